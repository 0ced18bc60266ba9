/* CPU timing harness for the reference library (test/bench infrastructure only).
 *
 * Modelled on the reference's single-thread loop (bench/bench.c:41-54): each
 * worker owns its own plans (a plan is not reentrant, docs/API.md:23) and calls
 * bridct_plan_apply once per array.  Work is split across T POSIX threads by
 * element count; plan creation happens before the timed region.  Loaded by
 * bench.py's CPU legs through ctypes; never part of the shipped library.
 */
#define _GNU_SOURCE
#include "bridct.h"
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <time.h>

typedef struct {
    size_t begin, end, repeats;
    const int *hs, *ws, *modes;
    const size_t *offsets;
    const float *input;
    float *output;
    bridct_plan *plans[8][8];
    int status;
    pthread_barrier_t *barrier;
} worker_t;

static int lg(int n) { int k = 0; while ((8 << k) < n) k++; return k; }

static void *work(void *arg)
{
    worker_t *w = arg;
    for (size_t i = w->begin; i < w->end; i++) {
        int a = lg(w->hs[i]), b = lg(w->ws[i]);
        if (!w->plans[a][b]) {
            w->plans[a][b] = bridct_plan_create(w->hs[i], w->ws[i]);
            if (!w->plans[a][b]) w->status = -100;
        }
    }
    pthread_barrier_wait(w->barrier);
    for (size_t r = 0; r < w->repeats && !w->status; r++)
        for (size_t i = w->begin; i < w->end; i++) {
            int s = bridct_plan_apply(w->plans[lg(w->hs[i])][lg(w->ws[i])],
                                      (enum bridct_mode)w->modes[i],
                                      w->input + w->offsets[i], w->output + w->offsets[i]);
            if (s) { w->status = s; break; }
        }
    pthread_barrier_wait(w->barrier);
    return NULL;
}

static double now(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* Runs `repeats` passes over `count` arrays with `threads` workers.
 * Returns elapsed seconds of the timed region, or a negative status. */
double ref_bench_run(size_t count, const int *hs, const int *ws, const int *modes,
                     const size_t *offsets, const float *input, float *output,
                     int threads, size_t repeats)
{
    if (threads < 1 || !count) return -1.0;
    if ((size_t)threads > count) threads = (int)count;
    worker_t *wk = calloc((size_t)threads, sizeof(worker_t));
    pthread_t *tid = calloc((size_t)threads, sizeof(pthread_t));
    pthread_barrier_t barrier;
    if (!wk || !tid) { free(wk); free(tid); return -2.0; }
    pthread_barrier_init(&barrier, NULL, (unsigned)threads + 1);
    double total = 0;
    for (size_t i = 0; i < count; i++) total += (double)hs[i] * ws[i];
    size_t pos = 0;
    double acc = 0;
    for (int t = 0; t < threads; t++) {
        wk[t].begin = pos;
        double target = total * (t + 1) / threads;
        while (pos < count && (acc < target || t == threads - 1)) {
            acc += (double)hs[pos] * ws[pos];
            pos++;
        }
        wk[t].end = pos;
        wk[t].repeats = repeats;
        wk[t].hs = hs; wk[t].ws = ws; wk[t].modes = modes; wk[t].offsets = offsets;
        wk[t].input = input; wk[t].output = output; wk[t].barrier = &barrier;
    }
    for (int t = 0; t < threads; t++) pthread_create(&tid[t], NULL, work, &wk[t]);
    pthread_barrier_wait(&barrier);
    double t0 = now();
    pthread_barrier_wait(&barrier);
    double t1 = now();
    int status = 0;
    for (int t = 0; t < threads; t++) {
        pthread_join(tid[t], NULL);
        if (wk[t].status) status = wk[t].status;
        for (int a = 0; a < 8; a++)
            for (int b = 0; b < 8; b++) bridct_plan_destroy(wk[t].plans[a][b]);
    }
    pthread_barrier_destroy(&barrier);
    free(wk); free(tid);
    return status ? (double)(status < 0 ? status : -status) - 1000.0 : t1 - t0;
}
