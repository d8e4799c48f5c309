/*
 * tpzh_search.c -- `topaz search` on the B200: the host part of
 * search_alloc/search_pthread (src/engine.c:38-87, :493-559) around the
 * device batch entry point tpz_search_batch.
 *
 * Per query, as the reference does it (src/engine.c:193-248,
 * src/ssw_wrapper.c:157-245, src/utils.c:140-152): every hit that was
 * aligned (SW score, or gapless score < 40 with bitscore 0 and E-value
 * 1000) in hitlist traversal order, stably sorted by bitscore descending,
 * the first -H of them, printed when the E-value is <= -E.  Bitscores and
 * E-values come from tpz_karlin (the C library's log/exp, same expression
 * order).  Queries print in input order; the reference prints them in
 * completion order of its threads, so parity is per-query block.
 *
 * -T N runs min(N, 4) host threads, each with one query batch on the device
 * at a time (the library runs every calling thread on its own CUDA stream),
 * so one batch's SW overlaps another's walk and the FASTA reading, SEG and
 * output formatting of the others.  Each batch formats its lines into a
 * buffer and the buffers are written in batch order.
 */
#define _GNU_SOURCE
#include "tpzh.h"
#include "../../include/topaz_b200.h"

#include <errno.h>
#include <time.h>
#include <fcntl.h>
#include <inttypes.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <unistd.h>

void tpzh_options_defaults(tpzh_options *o) {
    memset(o, 0, sizeof *o);
    o->num_threads = 1;
    o->num_hits = 100;
    o->evalue = 1e-3;
    o->gap_open = 11;
    o->gap_extend = 1;
    o->lambda = 0.267;
    o->k = 0.041;
    o->H = 0.140;
    o->matrix = "BLOSUM62";
    o->min_hit_length = 5;
    o->min_hit_score = 1;
    o->number_of_seeds = 300000;
    o->number_of_alignments = 5000;
    o->superfast = 1;
    o->seg_enabled = 1;
    o->batch = 2000;
}

typedef struct {
    const char *data;
    uint64_t size;
} map_t;

static int map_file(const char *prefix, const char *ext, map_t *m) {
    char name[4096];
    snprintf(name, sizeof name, "%s%s", prefix, ext);
    const int fd = open(name, O_RDONLY);
    struct stat sb;
    if (fd < 0 || fstat(fd, &sb) != 0) return -1;
    m->size = (uint64_t)sb.st_size;
    /* an empty file fails here with EINVAL, as fmmap_ro's mmap does
     * (src/utils.c:17-42) */
    m->data = mmap(NULL, m->size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m->data == MAP_FAILED) return -1;
    close(fd);
    return 0;
}

/* Page-table prefault of the text and SA mappings: threads touch one byte
 * per page while the CUDA context comes up, so the index upload that follows
 * copies from mapped pages instead of taking a fault per 4 KB page. */
#define TPZH_PREFAULT_THREADS 8
typedef struct {
    const volatile uint8_t *p;
    uint64_t n;
    uint64_t sum;
} prefault_t;

static void *prefault_thread(void *arg) {
    prefault_t *a = (prefault_t *)arg;
    uint64_t s = 0;
    for (uint64_t i = 0; i < a->n; i += 4096) s += a->p[i];
    a->sum = s;
    return NULL;
}

typedef struct {
    pthread_t th[2 * TPZH_PREFAULT_THREADS];
    prefault_t part[2 * TPZH_PREFAULT_THREADS];
    int started[2 * TPZH_PREFAULT_THREADS];
} prefault_set_t;

static void prefault_start(prefault_set_t *ps, const map_t *a, const map_t *b) {
    memset(ps, 0, sizeof *ps);
    const map_t *m[2] = {a, b};
    for (int f = 0; f < 2; ++f) {
        const uint64_t n = m[f]->size;
        const uint64_t chunk = ((n / TPZH_PREFAULT_THREADS) + 4095) & ~(uint64_t)4095;
        for (int t = 0; t < TPZH_PREFAULT_THREADS; ++t) {
            const uint64_t lo = (uint64_t)t * chunk;
            if (!chunk || lo >= n) break;
            const int k = f * TPZH_PREFAULT_THREADS + t;
            ps->part[k].p = (const volatile uint8_t *)m[f]->data + lo;
            ps->part[k].n = n - lo < chunk ? n - lo : chunk;
            ps->started[k] = pthread_create(&ps->th[k], NULL, prefault_thread, &ps->part[k]) == 0;
        }
    }
}

static void prefault_join(prefault_set_t *ps) {
    for (int k = 0; k < 2 * TPZH_PREFAULT_THREADS; ++k)
        if (ps->started[k]) pthread_join(ps->th[k], NULL);
    memset(ps->started, 0, sizeof ps->started);
}

typedef struct {
    int64_t idx;
    double bits, evalue;
} ranked_t;

/* stable by construction: insertion order breaks ties (glibc qsort is a
 * merge sort here, so equal bitscores keep traversal order) */
static void stable_sort_bits(ranked_t *v, int64_t n, ranked_t *tmp) {
    for (int64_t w = 1; w < n; w *= 2) {
        for (int64_t lo = 0; lo < n; lo += 2 * w) {
            int64_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            int64_t a = lo, b = mid, k = lo;
            while (a < mid && b < hi) tmp[k++] = (v[b].bits > v[a].bits) ? v[b++] : v[a++];
            while (a < mid) tmp[k++] = v[a++];
            while (b < hi) tmp[k++] = v[b++];
        }
        memcpy(v, tmp, sizeof(ranked_t) * n);
    }
}

static int8_t g_int2idx[128];

static void init_int2idx(void) {
    static const char order[] = "ACMLJIVTSKRQZEDBNHYFWXP*G";
    static const char mat[] = "ARNDCQEGHILKMFPSTWYVBJZX*";
    for (int i = 0; i < 128; ++i) g_int2idx[i] = 23;
    for (int i = 0; i < 25; ++i) g_int2idx['A' + i] = (int8_t)(strchr(mat, order[i]) - mat);
}

typedef struct {
    char *id;
    int id_len;
    char *seq;      /* internal alphabet */
    int len;
} query_t;

typedef struct { uint64_t hs, ps; int32_t hl, pl; } rec_t;

#define TPZH_MAX_WORKERS 4

/* What the worker threads of one `topaz search` share. */
typedef struct {
    const tpzh_options *o;
    tpz_index *ix;
    const tpz_search_opts *so;
    int report;
    const int8_t *mat;
    const rec_t *recs;
    const char *T, *phr;
    uint64_t db_size, db_proteins;
    int64_t B;
    int prep_threads;
    tpzh_fasta *f;
    pthread_mutex_t mu;         /* the reader, the print turn and the totals */
    pthread_cond_t turn;
    int64_t next_read, next_print;
    int done;
    uint64_t nonzero, total_hits;
    /* time spent, summed over batches (under mu): device stages of
     * tpz_search_batch (seed + chains, walk + hitlist, SW + ranking), the
     * batch calls' wall time, host ingest (SEG + alphabet) and formatting */
    double dev_ms[3], call_s, ingest_s, format_s;
} search_ctx;

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

/* A --blasttab line: query, hit, ranking values and its statistics. */
typedef struct {
    int64_t q, h;
    double bits, evalue;
    tpzh_stats st;
} line_t;

typedef struct {
    const search_ctx *c;
    const query_t *qs;
    const tpz_search_result *res;
    line_t *lines;
    int64_t from, to;
} stats_job;

/* ssw_align_stats (src/ssw_wrapper.c:132-155) of the lines [from, to): one
 * host thread's share of a batch. */
static void *stats_worker(void *arg) {
    const stats_job *j = arg;
    const search_ctx *c = j->c;
    const tpz_search_result *res = j->res;
    for (int64_t i = j->from; i < j->to; ++i) {
        line_t *ln = &j->lines[i];
        const int64_t h = ln->h;
        memset(&ln->st, 0, sizeof ln->st);
        if (res->sw_status[h] == TPZ_SW_OK) {
            const query_t *qq = &j->qs[ln->q];
            const rec_t *pr = &c->recs[res->protein[h]];
            int8_t *qidx = malloc(qq->len + 1), *sidx = malloc(pr->pl + 1);
            for (int k = 0; k < qq->len; ++k) qidx[k] = g_int2idx[(int)qq->seq[k] & 127];
            for (int k = 0; k < pr->pl; ++k) sidx[k] = g_int2idx[(int)c->T[pr->ps + k] & 127];
            tpzh_align_stats(qidx, qq->len, sidx, pr->pl, c->mat, c->o->gap_open, c->o->gap_extend,
                             res->qend[h], res->send[h], res->rawscore[h], &ln->st);
            free(qidx);
            free(sidx);
        } else {
            ln->st.qstart = ln->st.sstart = -1;
            ln->st.length = ln->st.mismatch = ln->st.gapopen = -1;
            ln->st.identity = INFINITY;
        }
    }
    return NULL;
}

/* One batch: SEG + alphabet, the device search, then the lines of every
 * query into `out`.  --blasttab statistics (about a millisecond per line)
 * are computed for the whole batch over host threads before printing. */
static void search_batch(search_ctx *c, query_t *qs, int64_t nq, FILE *out, uint64_t *nonzero,
                         uint64_t *total_hits) {
    const tpzh_options *o = c->o;
    const int report = c->report;
    int64_t total = 0;
    int64_t *qoff = malloc(sizeof(int64_t) * nq);
    int32_t *qlen = malloc(sizeof(int32_t) * nq);
    for (int64_t i = 0; i < nq; ++i) { qoff[i] = total; qlen[i] = qs[i].len; total += qs[i].len; }
    char *cat = malloc(total + 1);
    for (int64_t i = 0; i < nq; ++i) memcpy(cat + qoff[i], qs[i].seq, qs[i].len);
    /* run_seg + seq_2internal: on the device inside the batch call when the
     * statistics are computed there too (report mode), else over host
     * threads (the host statistics read the prepared queries) */
    const double t_in = now_s();
    tpz_search_opts so = *c->so;
    if (c->report) {
        so.ingest = o->seg_enabled ? 1 : 2;
    } else {
        tpz_prepare_queries(cat, qoff, qlen, nq, o->seg_enabled, c->prep_threads);
        for (int64_t i = 0; i < nq; ++i) memcpy(qs[i].seq, cat + qoff[i], qs[i].len);
    }
    tpz_search_result *res = NULL;
    const double t_call = now_s();
    if (tpz_search_batch(c->ix, cat, qoff, qlen, nq, &so, &res) != 0) {
        fprintf(stderr, "Error: %s\n", tpz_last_error());
        exit(EXIT_FAILURE);
    }
    const double t_fmt = now_s();
    pthread_mutex_lock(&c->mu);
    for (int k = 0; k < 3; ++k) c->dev_ms[k] += res->stage_ms[k];
    c->ingest_s += t_call - t_in;
    c->call_s += t_fmt - t_call;
    pthread_mutex_unlock(&c->mu);
    int64_t maxh = 1;
    for (int64_t q = 0; q < nq; ++q) {
        const int64_t nh = res->hit_off[q + 1] - res->hit_off[q];
        if (nh > maxh) maxh = nh;
    }
    ranked_t *rk = malloc(sizeof(ranked_t) * maxh), *tmp = malloc(sizeof(ranked_t) * maxh);
    line_t *lines = NULL;
    int64_t nlines = 0, lcap = 0;
    for (int64_t q = 0; q < nq; ++q) {
        if (res->status[q] & TPZ_Q_SA_END)
            fprintf(stderr, "Warning: %.*s reached the end of the suffix array (the reference reads past its mapping there)\n",
                    qs[q].id_len, qs[q].id);
        const int64_t a = res->hit_off[q], b = res->hit_off[q + 1];
        int64_t n = 0;
        if (report) {
            /* already ranked, cut to -H and to -E */
            for (int64_t h = a; h < b; ++h) {
                rk[n].idx = h; rk[n].bits = res->bitscore[h]; rk[n].evalue = res->evalue[h]; n++;
            }
        } else
        for (int64_t h = a; h < b; ++h) {
            const int st = res->sw_status[h];
            if (st == TPZ_SW_OK) {
                rk[n].idx = h;
                tpz_karlin(qs[q].len, c->db_size, c->db_proteins, o->lambda, o->k, o->H, res->rawscore[h],
                           &rk[n].bits, &rk[n].evalue);
                n++;
            } else if (st == TPZ_SW_GAPLESS_LOW) {
                rk[n].idx = h; rk[n].bits = 0; rk[n].evalue = 1000; n++;
            }
        }
        if (!report) {
            stable_sort_bits(rk, n, tmp);
            if (n > o->num_hits) n = o->num_hits;
        }
        int count = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (!(rk[i].evalue <= o->evalue)) continue;
            const int64_t h = rk[i].idx;
            if (o->superfast) {
                const rec_t *pr = &c->recs[res->protein[h]];
                const char *sid;
                const int sl = tpzh_header_id(c->phr + pr->hs, pr->hl, &sid);
                fprintf(out, "%.*s\t%.*s\t%.3e\t%d\n", qs[q].id_len, qs[q].id, sl, sid, rk[i].evalue,
                        (int)rk[i].bits);
            } else {
                if (nlines == lcap) {
                    lcap = lcap ? 2 * lcap : 1024;
                    lines = realloc(lines, sizeof(line_t) * lcap);
                    if (!lines) { fprintf(stderr, "Error: out of memory\n"); exit(EXIT_FAILURE); }
                }
                line_t *ln = &lines[nlines++];
                ln->q = q; ln->h = h; ln->bits = rk[i].bits; ln->evalue = rk[i].evalue;
            }
            ++count;
        }
        if (count) { (*nonzero)++; *total_hits += count; }
    }
    if (nlines && res->qstart) {
        /* the statistics came with the batch (computed on the device) */
        for (int64_t i = 0; i < nlines; ++i) {
            line_t *ln = &lines[i];
            const int64_t h = ln->h;
            ln->st.qstart = res->qstart[h];
            ln->st.sstart = res->sstart[h];
            ln->st.length = res->length[h];
            ln->st.mismatch = res->mismatch[h];
            ln->st.gapopen = res->gapopen[h];
            ln->st.identity = res->sw_status[h] == TPZ_SW_OK ? res->identity[h] : INFINITY;
        }
    } else if (nlines) {
        /* statistics over host threads, then the lines in order */
        int nt = c->prep_threads < 1 ? 1 : c->prep_threads;
        if (nt > nlines) nt = (int)nlines;
        stats_job jobs[64];
        pthread_t th[64];
        int running[64] = {0};
        if (nt > 64) nt = 64;
        const int64_t per = (nlines + nt - 1) / nt;
        for (int t = 0; t < nt; ++t) {
            jobs[t].c = c; jobs[t].qs = qs; jobs[t].res = res; jobs[t].lines = lines;
            jobs[t].from = t * per < nlines ? t * per : nlines;
            jobs[t].to = (t + 1) * per < nlines ? (t + 1) * per : nlines;
        }
        for (int t = 1; t < nt; ++t) {
            running[t] = pthread_create(&th[t], NULL, stats_worker, &jobs[t]) == 0;
            if (!running[t]) stats_worker(&jobs[t]);
        }
        stats_worker(&jobs[0]);
        for (int t = 1; t < nt; ++t)
            if (running[t]) pthread_join(th[t], NULL);
    }
    if (nlines) {
        for (int64_t i = 0; i < nlines; ++i) {
            const line_t *ln = &lines[i];
            const int64_t q = ln->q, h = ln->h;
            const rec_t *pr = &c->recs[res->protein[h]];
            const char *sid;
            const int sl = tpzh_header_id(c->phr + pr->hs, pr->hl, &sid);
            const tpzh_stats *st = &ln->st;
            fprintf(out, "%.*s\t%.*s\t%.2f\t%d\t%d\t%d\t%d\t%d\t%d\t%d\t%.3e\t%d\n", qs[q].id_len,
                    qs[q].id, sl, sid, st->identity * 100, st->length, st->mismatch, st->gapopen,
                    st->qstart + 1, res->qend[h] + 1, st->sstart + 1, res->send[h] + 1, ln->evalue,
                    (int)ln->bits);
        }
    }
    free(lines);
    free(rk); free(tmp);
    tpz_search_result_free(res);
    free(cat); free(qoff); free(qlen);
    pthread_mutex_lock(&c->mu);
    c->format_s += now_s() - t_fmt;
    pthread_mutex_unlock(&c->mu);
}

/* Worker: take the next batch from the FASTA reader (batch ids in reading
 * order), search and format it, then write it when every earlier batch has
 * been written. */
static void *search_worker(void *arg) {
    search_ctx *c = arg;
    query_t *qs = calloc(c->B, sizeof(query_t));
    for (;;) {
        int64_t nq = 0, id = -1;
        pthread_mutex_lock(&c->mu);
        while (!c->done && nq < c->B) {
            tpzh_record r;
            const int rc = tpzh_fasta_next(c->f, &r);
            if (rc < 0) exit(EXIT_FAILURE);
            if (rc == 0) { c->done = 1; break; }
            qs[nq].id = r.id; qs[nq].id_len = r.id_len;
            qs[nq].seq = r.seq; qs[nq].len = r.seq_len;
            nq++;
        }
        if (nq) id = c->next_read++;
        pthread_mutex_unlock(&c->mu);
        if (nq == 0) break;
        char *buf = NULL;
        size_t len = 0;
        FILE *out = open_memstream(&buf, &len);
        if (!out) { fprintf(stderr, "Error: %s\n", strerror(errno)); exit(EXIT_FAILURE); }
        uint64_t nonzero = 0, total_hits = 0;
        search_batch(c, qs, nq, out, &nonzero, &total_hits);
        fclose(out);
        for (int64_t i = 0; i < nq; ++i) { free(qs[i].id); free(qs[i].seq); }
        pthread_mutex_lock(&c->mu);
        while (c->next_print != id) pthread_cond_wait(&c->turn, &c->mu);
        fwrite(buf, 1, len, stdout);
        c->next_print++;
        c->nonzero += nonzero;
        c->total_hits += total_hits;
        pthread_cond_broadcast(&c->turn);
        pthread_mutex_unlock(&c->mu);
        free(buf);
    }
    free(qs);
    return NULL;
}

static void *device_init_thread(void *arg) {
    *(int *)arg = tpz_device_init();
    return NULL;
}

/* the start-up thread is joined before the process ends on any path */
static pthread_t g_init_th;
static int g_init_started, g_init_rc;
static void join_init(void) {
    if (g_init_started) pthread_join(g_init_th, NULL);
    g_init_started = 0;
}

int tpzh_search(const char *fasta, const char *prefix, const tpzh_options *o) {
    struct timeval t0, t1;
    gettimeofday(&t0, NULL);
    const double t_start = now_s();
    /* the CUDA context comes up while the database files are mapped */
    g_init_started = pthread_create(&g_init_th, NULL, device_init_thread, &g_init_rc) == 0;
    /* db_load / _load_index (src/db.c:34-122) in the same order, with the
     * same messages; a file that cannot be mapped ends the process with
     * engine_init's message (src/engine.c:47-50) */
    map_t T, SA, phr, ind;
    if (map_file(prefix, ".psq", &T)) goto load_fail;
    fprintf(stderr, "read T (%s.psq), file size is %" PRIu64 " bytes\n", prefix, T.size);
    if (map_file(prefix, ".SA", &SA)) goto load_fail;
    fprintf(stderr, "read SA (%s.SA), file size is %" PRIu64 " bytes\n", prefix, SA.size);
    if (SA.size != T.size * 8) {
        fprintf(stderr, "Error: SA (%s.SA, %" PRIu64 " bytes) should be 8 x T (%s.psq, %" PRIu64 " bytes)!\nExiting...\n",
                prefix, SA.size, prefix, T.size);
        join_init();
        exit(EXIT_FAILURE);
    }
    if (map_file(prefix, ".phr", &phr)) goto load_fail;
    fprintf(stderr, "read protein headers (%s.phr), file size is %" PRIu64 " bytes\n", prefix, phr.size);
    uint64_t Psize = 0;
    for (uint64_t i = 0; i < phr.size; ++i) {
        if (phr.data[i] == '\0') break;
        if (phr.data[i] == '\n') Psize++;
    }
    fprintf(stderr, "%" PRIu64 " proteins in database\n", Psize);
    if (map_file(prefix, ".ind", &ind)) {
        fprintf(stderr, "Error: could not open %s.ind, %s\n", prefix, strerror(errno));
        goto load_fail;
    }
    if (ind.size != Psize * 24) {
        fprintf(stderr, "Error: index is the wrong size (read %" PRIu64 ", expected %" PRIu64 ")", ind.size, Psize * 24);
        join_init();
        exit(EXIT_FAILURE);
    }
    if (0) {
load_fail:
        fprintf(stderr, "Error: could not load database, %s\n", strerror(errno));
        join_init();
        exit(EXIT_FAILURE);
    }
    const uint64_t db_size = T.size - Psize, db_proteins = Psize;
    fprintf(stderr, "db size = %" PRIu64 "\n", db_size);
    fprintf(stderr, "db proteins = %" PRIu64 "\n", db_proteins);

    int8_t mat[625];
    if (tpz_matrix(o->matrix, mat) != 0) {
        fprintf(stderr, "Error: %s\n", tpz_last_error());
        join_init();
        return -1;
    }
    const double t_map = now_s();
    prefault_set_t pf;
    prefault_start(&pf, &T, &SA);
    join_init();
    const double init_wait_s = now_s() - t_map;
    prefault_join(&pf);
    const double prefault_wait_s = now_s() - t_map - init_wait_s;
    if (g_init_rc != 0 && tpz_device_init() != 0) {   /* again here, for this thread's message */
        fprintf(stderr, "Error: %s\n", tpz_last_error());
        return -1;
    }
    tpz_index *ix = NULL;
    const double t_up = now_s();
    if (tpz_index_create((const uint8_t *)T.data, (int64_t)T.size, (const int64_t *)SA.data, ind.data,
                         (int64_t)Psize, &ix) != 0) {
        fprintf(stderr, "Error: %s\n", tpz_last_error());
        return -1;
    }
    const double upload_s = now_s() - t_up;
    const double t_search = now_s();
    const rec_t *recs = (const rec_t *)ind.data;
    init_int2idx();

    if (o->superfast) printf("qseqid sseqid evalue bitscore\n");
    else printf("qseqid sseqid pident length mismatch gapopen qstart qend sstart send evalue bitscore\n");

    tpzh_fasta f;
    if (tpzh_fasta_open(&f, fasta) != 0) exit(EXIT_FAILURE);
    tpz_search_opts so;
    memset(&so, 0, sizeof so);
    so.num_hits = o->num_hits;
    so.gap_open = o->gap_open;
    so.gap_extend = o->gap_extend;
    so.min_hit_length = o->min_hit_length;
    so.seeds = o->number_of_seeds;
    so.alignments = o->number_of_alignments;
    so.mat625 = mat;
    /* ranking and the E-value cut on the device (report mode) unless the
     * Karlin parameters are outside what it takes (k <= 0, NaN -E) */
    const int report = o->k > 0 && o->evalue == o->evalue;
    if (report) {
        /* --blasttab columns of the printed hits on the device */
        so.blasttab_stats = o->superfast ? 0 : 1;
        so.report_hits = o->num_hits;
        so.max_evalue = o->evalue;
        so.lambda = o->lambda;
        so.k = o->k;
        so.H = o->H;
        so.db_size = db_size;
        so.db_proteins = db_proteins;
    }
    int nw = o->num_threads < 1 ? 1 : o->num_threads;
    if (nw > TPZH_MAX_WORKERS) nw = TPZH_MAX_WORKERS;
    const long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    search_ctx c;
    memset(&c, 0, sizeof c);
    c.o = o; c.ix = ix; c.so = &so; c.report = report; c.mat = mat; c.recs = recs;
    c.T = T.data; c.phr = phr.data; c.db_size = db_size; c.db_proteins = db_proteins;
    c.B = o->batch > 0 ? o->batch : 2000;
    c.prep_threads = ncpu > nw ? (int)(ncpu / nw) : 1;
    c.f = &f;
    pthread_mutex_init(&c.mu, NULL);
    pthread_cond_init(&c.turn, NULL);
    pthread_t th[TPZH_MAX_WORKERS];
    for (int i = 1; i < nw; ++i)
        if (pthread_create(&th[i], NULL, search_worker, &c) != 0) {
            fprintf(stderr, "Error: could not start a search thread\n");
            exit(EXIT_FAILURE);
        }
    search_worker(&c);
    for (int i = 1; i < nw; ++i) pthread_join(th[i], NULL);
    pthread_cond_destroy(&c.turn);
    pthread_mutex_destroy(&c.mu);
    const uint64_t nonzero = c.nonzero, total_hits = c.total_hits;
    fflush(stdout);
    tpzh_fasta_close(&f);
    const double t_end = now_s();
    tpz_index_destroy(ix);
    const double destroy_s = now_s() - t_end;
    gettimeofday(&t1, NULL);
    fprintf(stderr, "output %" PRIu64 " hits for %" PRIu64 " queries\n", total_hits, nonzero);
    fprintf(stderr, "timing: files mapped %.2f s, device init wait %.2f s, page prefault wait "
            "%.2f s, index upload %.2f s, queries %.2f s (%d host threads; summed over batches: "
            "ingest %.2f s, batch calls %.2f s, format %.2f s; device seed %.0f ms, walk %.0f ms, "
            "SW + ranking %.0f ms), index release %.2f s\n",
            t_map - t_start, init_wait_s, prefault_wait_s, upload_s, t_end - t_search, nw,
            c.ingest_s, c.call_s, c.format_s, c.dev_ms[0], c.dev_ms[1], c.dev_ms[2], destroy_s);
    fprintf(stderr, "elapsed time: %.1f seconds\n",
            ((t1.tv_sec - t0.tv_sec) * 1000.0 + (t1.tv_usec - t0.tv_usec) / 1000.0) / 1000);
    fprintf(stderr, "done!\n");
    return 0;
}
