/* ora_threads.h -- TEST INFRASTRUCTURE ONLY: a dynamic parallel-for over
 * [0, total) on POSIX threads, used by the oracle's CPU loops. */
#ifndef ORA_THREADS_H
#define ORA_THREADS_H
#include <pthread.h>
#include <unistd.h>

typedef void (*ora_body)(long long i, void *ctx, long long *acc);

typedef struct {
    long long total, chunk, next, acc;
    ora_body body;
    void *ctx;
    pthread_mutex_t mu;
} ora_pool;

static void *ora_worker(void *arg)
{
    ora_pool *p = (ora_pool *)arg;
    long long local = 0;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        long long lo = p->next;
        p->next += p->chunk;
        pthread_mutex_unlock(&p->mu);
        if (lo >= p->total) break;
        long long hi = lo + p->chunk < p->total ? lo + p->chunk : p->total;
        for (long long i = lo; i < hi; i++) p->body(i, p->ctx, &local);
    }
    pthread_mutex_lock(&p->mu);
    p->acc += local;
    pthread_mutex_unlock(&p->mu);
    return NULL;
}

/* Runs body(i) for every i in [0, total) on nthreads threads (<= 0: all
 * online cores); returns the sum of what the bodies added to *acc. */
static long long ora_parallel_for(long long total, int nthreads, long long chunk,
                                  ora_body body, void *ctx)
{
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    ora_pool p;
    p.total = total; p.chunk = chunk > 0 ? chunk : 1; p.next = 0; p.acc = 0;
    p.body = body; p.ctx = ctx;
    pthread_mutex_init(&p.mu, NULL);
    pthread_t th[256];
    int started = 0;
    for (int t = 1; t < nthreads; t++)
        if (pthread_create(&th[started], NULL, ora_worker, &p) == 0) started++;
    ora_worker(&p);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&p.mu);
    return p.acc;
}
#endif
