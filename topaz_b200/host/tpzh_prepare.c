/*
 * tpzh_prepare.c -- query ingest for a batch (run_seg + seq_2internal,
 * src/engine.c:250-277): SEG hard-masking, then the internal alphabet, in
 * place, over host threads.
 */
#include "tpzh.h"
#include "../../include/topaz_b200.h"

#include <pthread.h>
#include <stdlib.h>

typedef struct {
    char *cat;
    const int64_t *off;
    const int32_t *len;
    int64_t lo, hi;
    int seg;
} prep_job;

static void *prep_work(void *p) {
    prep_job *j = (prep_job *)p;
    for (int64_t i = j->lo; i < j->hi; ++i) {
        char *s = j->cat + j->off[i];
        if (j->seg) tpzh_seg_mask(s, j->len[i]);
        for (int32_t k = 0; k < j->len[i]; ++k) s[k] = tpzh_aa2internal(s[k]);
    }
    return NULL;
}

int tpz_prepare_queries(char *cat, const int64_t *off, const int32_t *len, int64_t n, int seg,
                        int nthreads) {
    if (n < 0 || (n > 0 && (!cat || !off || !len))) return TPZ_E_ARG;
    for (int64_t i = 0; i < n; ++i)
        if (len[i] < 0 || off[i] < 0) return TPZ_E_ARG;
    if (n == 0) return TPZ_OK;
    if (seg) {
        char x = 'A';
        tpzh_seg_mask(&x, 0);          /* the one-time SEG tables, before the threads */
    }
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 64) nthreads = 64;
    if (nthreads > n) nthreads = (int)n;
    prep_job jobs[64];
    pthread_t th[64];
    int running[64] = {0};
    for (int t = 0; t < nthreads; ++t) {
        jobs[t].cat = cat; jobs[t].off = off; jobs[t].len = len; jobs[t].seg = seg;
        jobs[t].lo = n * t / nthreads;
        jobs[t].hi = n * (t + 1) / nthreads;
    }
    for (int t = 1; t < nthreads; ++t)
        running[t] = pthread_create(&th[t], NULL, prep_work, &jobs[t]) == 0;
    prep_work(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) {
        if (running[t]) pthread_join(th[t], NULL);
        else prep_work(&jobs[t]);                  /* no thread: do it here */
    }
    return TPZ_OK;
}
