/* Batched solves of independent problems (the C5 sweep of many small dots).
 *
 * Each instance is a full solve (tables, assembly, windowed eigensolve).  One
 * small instance cannot fill the GPU: most of its kernels are latency-bound
 * (panel factorisations, bulge chasing, inverse iteration).  The batch
 * therefore runs several solves at once, one per host thread, each on the
 * thread's own default stream (the library is built with per-thread default
 * streams and a cuBLAS handle per thread), taking instances largest first
 * from a shared queue. */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "qd_internal.h"

typedef struct {
    qd_problem **pr;
    int n, prec, device;
    double *const *eigval;
    qd_complex128 *const *eigvec;
    int *order;
    int next;
    int sm_share; /* SMs each worker's solves spread over (0: the whole GPU) */
    int rc;
    char msg[512];
    pthread_mutex_t mu;
} batch_queue;

static void *batch_worker(void *arg) {
    batch_queue *q = (batch_queue *)arg;
    cudaSetDevice(q->device);
    qd_set_sm_budget(q->sm_share);
    for (;;) {
        pthread_mutex_lock(&q->mu);
        int k = (q->rc == QD_OK && q->next < q->n) ? q->order[q->next++] : -1;
        pthread_mutex_unlock(&q->mu);
        if (k < 0) break;
        int rc = qd_problem_solve(q->pr[k], q->prec, q->eigval[k], q->eigvec[k]);
        if (rc != QD_OK) {
            pthread_mutex_lock(&q->mu);
            if (q->rc == QD_OK) {
                q->rc = rc;
                strncpy(q->msg, qd_last_error_message(), sizeof(q->msg) - 1);
            }
            pthread_mutex_unlock(&q->mu);
        }
    }
    qd_set_sm_budget(0);
    return NULL;
}

static int by_size_desc(const void *a, const void *b, void *ctx) {
    qd_problem **pr = (qd_problem **)ctx;
    int64_t na = pr[*(const int *)a]->n_h, nb = pr[*(const int *)b]->n_h;
    return na < nb ? 1 : na > nb ? -1 : 0;
}

int eigenstates_batched(qd_problem **problems, int n, int prec, int n_threads, double *const *eigval,
                        qd_complex128 *const *eigvec) {
    if (!problems || n < 1 || !eigval || !eigvec) return qd_set_error(QD_ERR_ARG, "eigenstates_batched: bad arguments");
    if (n_threads < 1) n_threads = 1;
    if (n_threads > n) n_threads = n;
    batch_queue q;
    memset(&q, 0, sizeof(q));
    q.pr = problems;
    q.n = n;
    q.prec = prec;
    q.eigval = eigval;
    q.eigvec = eigvec;
    q.order = (int *)malloc(sizeof(int) * (size_t)n);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)n_threads);
    if (!q.order || !th) {
        free(q.order);
        free(th);
        return qd_set_error(QD_ERR_NOMEM, "eigenstates_batched");
    }
    for (int i = 0; i < n; i++) q.order[i] = i;
    qsort_r(q.order, (size_t)n, sizeof(int), by_size_desc, problems);
    cudaGetDevice(&q.device);
    /* Each worker's kernels spread over a share of the SMs (twice the even
     * split, at least 16), so that the latency-bound stages of several
     * instances run side by side instead of queueing behind kernels that take
     * the whole GPU.  QD_BATCH_SMS overrides it (0: the whole GPU). */
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, q.device);
    q.sm_share = n_threads > 1 ? 2 * nsm / n_threads : 0;
    if (q.sm_share && q.sm_share < 16) q.sm_share = 16;
    const char *env = getenv("QD_BATCH_SMS");
    if (env) q.sm_share = atoi(env) > 0 ? atoi(env) : 0;
    pthread_mutex_init(&q.mu, NULL);
    /* handles of the threads that did start are kept contiguous, so only those are joined */
    int started = 0;
    for (int t = 0; t < n_threads; t++) {
        pthread_t tid;
        if (pthread_create(&tid, NULL, batch_worker, &q) == 0) th[started++] = tid;
    }
    if (started == 0) batch_worker(&q); /* no threads available: run in the caller */
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&q.mu);
    free(q.order);
    free(th);
    if (q.rc != QD_OK) return qd_set_error(q.rc, "eigenstates_batched: %s", q.msg);
    return QD_OK;
}
