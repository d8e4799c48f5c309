/*
 * ref_driver.c -- stage-level drivers around the UNMODIFIED TOPAZ sources.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
 * reference's own src/*.c files (see oracle/Makefile) into
 * oracle/_ref/libtopazref.so.  It is used to pin the CPU restatement in
 * oracle/oracle.c and as the timed "reference" CPU baseline.  Nothing in the
 * product links it.
 *
 * Every function below only builds the reference's own structures (db_t,
 * seq_t, options_t) from flat buffers and then calls the reference's own
 * functions in the order the reference calls them:
 *   - ssw_init / ssw_align / ssw_align_stats      src/ssw.c:799, :835, :900
 *   - sa_search / sa_hsp                           src/search.c:237, :99
 *   - query_find_suffixes, the pqueue_next/hitlist_add loop of
 *     query_fetch_alignment_batch, query_perform_alignments,
 *     query_perform_statistics                     src/query.c:94-299
 *   - initialise_seg / run_seg                     src/seg_wrapper.c:11-49
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include "db.h"
#include "hit.h"
#include "options.h"
#include "priority_queue.h"
#include "query.h"
#include "search.h"
#include "seg_wrapper.h"
#include "seq.h"
#include "ssw.h"
#include "ssw_wrapper.h"
#include "substitution.h"
#include "lexicographical.h"

/* ------------------------------------------------------------------ SW */

/* One pair through ssw_init(score_size=2) + ssw_align exactly as
 * align_using_ssw_profile does (src/ssw_wrapper.c:209-217).
 * Returns 0 and fills score/ref_end/read_end, or 1 when ssw_align returned
 * NULL (word overflow, hit dropped by the caller). */
int ref_ssw_align(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                  const int8_t *mat25, int gap_open, int gap_extend,
                  int32_t *score, int32_t *ref_end, int32_t *read_end) {
    s_profile *p = ssw_init(q, qlen, mat25, 25, 2);
    s_align *a = ssw_align(p, s, slen, (uint8_t)gap_open, (uint8_t)gap_extend, 0, 0, 0, 15);
    int rc = 0;
    if (a == NULL) {
        rc = 1;
        *score = 32767; *ref_end = -1; *read_end = -1;
    } else {
        *score = a->score1; *ref_end = a->ref_end1; *read_end = a->read_end1;
        align_destroy(a);
    }
    init_destroy(p);
    return rc;
}

typedef struct {
    const int8_t *q; const int64_t *qoff; const int32_t *qlen;
    const int8_t *s; const int64_t *soff; const int32_t *slen;
    const int8_t *mat; int go, ge;
    int32_t *score, *ref_end, *read_end, *status;
    int64_t n, t, nt;
} batch_arg_t;

static void *batch_worker(void *v) {
    batch_arg_t *b = (batch_arg_t *)v;
    for (int64_t i = b->t; i < b->n; i += b->nt) {
        b->status[i] = ref_ssw_align(b->q + b->qoff[i], b->qlen[i], b->s + b->soff[i], b->slen[i],
                                     b->mat, b->go, b->ge, &b->score[i], &b->ref_end[i], &b->read_end[i]);
    }
    return NULL;
}

/* Pairs i in [0,n): query q[qoff[i] .. +qlen[i]), subject s[soff[i] .. +slen[i]),
 * both as matrix indices.  One ssw_init per pair (every pair has its own
 * query), split over nthreads pthreads. */
void ref_ssw_batch(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                   const int8_t *s, const int64_t *soff, const int32_t *slen,
                   const int8_t *mat25, int go, int ge, int nthreads,
                   int32_t *score, int32_t *ref_end, int32_t *read_end, int32_t *status) {
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = malloc(sizeof(pthread_t) * nthreads);
    batch_arg_t *args = malloc(sizeof(batch_arg_t) * nthreads);
    for (int t = 0; t < nthreads; ++t) {
        batch_arg_t a = {q, qoff, qlen, s, soff, slen, mat25, go, ge, score, ref_end, read_end, status, n, t, nthreads};
        args[t] = a;
        pthread_create(&th[t], NULL, batch_worker, &args[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th); free(args);
}

/* ssw_align_stats for a hit whose forward pass gave (score1, read_end1,
 * ref_end1) (src/ssw.c:900-978). */
int ref_ssw_stats(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                  const int8_t *mat25, int go, int ge,
                  int32_t read_end1, int32_t ref_end1, int32_t score1,
                  int32_t *read_begin1, int32_t *ref_begin1, int32_t *length,
                  int32_t *gapopen, int32_t *mismatch, double *identity) {
    int8_t *qcopy = malloc(qlen > 0 ? qlen : 1);
    memcpy(qcopy, q, qlen);
    s_profile *p = ssw_init(qcopy, qlen, mat25, 25, 2);
    int rc = ssw_align_stats(p, s, slen, (uint8_t)go, (uint8_t)ge, 15, read_end1, ref_end1,
                             (uint16_t)score1, read_begin1, ref_begin1, length, gapopen,
                             mismatch, identity);
    init_destroy2(p);  /* frees qcopy too */
    return rc;
}

/* ------------------------------------------------------------------ DB */

typedef struct {
    db_t db;
    int64_t *sa_padded;
} ref_db_t;

/* Build a db_t over caller-owned buffers.  The SA is copied into a buffer
 * padded with zero entries up to the next 4 KiB boundary plus one extra
 * zero page, which is what an mmap of the .SA file reads past its end
 * (src/db.c:362 maps the file; search.c:100 and hit.c:138 read SA[Tsize]). */
void *ref_db_open(const char *T, uint64_t Tsize, const int64_t *SA,
                  const void *ind, uint64_t Psize, const char *headers, uint64_t Hsize) {
    ref_db_t *r = calloc(1, sizeof(ref_db_t));
    uint64_t bytes = Tsize * 8;
    uint64_t padded = ((bytes + 4095) / 4096) * 4096 + 4096;
    r->sa_padded = calloc(padded / 8, 8);
    memcpy(r->sa_padded, SA, bytes);
    r->db.prefix = strdup("mem");
    r->db.headers = (char *)headers;
    r->db.Hsize = Hsize;
    r->db.index = (position_t *)ind;
    r->db.Psize = Psize;
    r->db.T = (char *)T;
    r->db.Tsize = Tsize;
    r->db.SA = r->sa_padded;
    r->db.SAsize = bytes;
    return r;
}

void ref_db_close(void *h) {
    ref_db_t *r = (ref_db_t *)h;
    if (!r) return;
    free(r->db.prefix);
    free(r->sa_padded);
    free(r);
}

static const char *MATNAMES[] = {"BLOSUM45", "BLOSUM50", "BLOSUM62", "BLOSUM80", "BLOSUM90",
                                 "PAM30", "PAM70", "PAM250", NULL};

/* Matrix table in the reference's 25x25 ARNDCQEGHILKMFPSTWYVBJZX* order. */
const int8_t *ref_matrix(const char *name) {
    if (!strcmp(name, "BLOSUM45")) return BLOSUM45;
    if (!strcmp(name, "BLOSUM50")) return BLOSUM50;
    if (!strcmp(name, "BLOSUM62")) return BLOSUM62;
    if (!strcmp(name, "BLOSUM80")) return BLOSUM80;
    if (!strcmp(name, "BLOSUM90")) return BLOSUM90;
    if (!strcmp(name, "PAM30")) return PAM30;
    if (!strcmp(name, "PAM70")) return PAM70;
    if (!strcmp(name, "PAM250")) return PAM250;
    return NULL;
}

const char *ref_matrix_name(int i) { return MATNAMES[i]; }

/* aa_table2 (src/lexicographical.h:19-33): internal letter -> matrix index. */
int ref_aa_table2(int c) { return aa_table2[c & 127]; }
/* aa2internal (src/lexicographical.h:135-192). */
int ref_aa2internal(int c) { return aa2internal((char)c); }
/* upper_aa (src/lexicographical.h:35-58). */
int ref_upper_aa(int c) { return upper_aa((char)c); }

static void set_options(options_t *o, const ref_db_t *r, const char *matrix, int num_hits,
                        double evalue, int go, int ge, double lambda, double k, double H,
                        int min_hit_length, int seeds, int alignments, int superfast) {
    memset(o, 0, sizeof(*o));
    o->num_threads = 1;
    o->num_hits = num_hits;
    o->evalue = evalue;
    o->gap_open = go;
    o->gap_extend = ge;
    o->sub_name = (char *)matrix;
    o->substitution = (int8_t (*)[625])ref_matrix(matrix);
    o->db_size = r->db.Tsize - r->db.Psize;      /* src/engine.c:53 */
    o->db_proteins = r->db.Psize;
    o->lambda = lambda;
    o->k = k;
    o->H = H;
    o->min_hit_length = min_hit_length;
    o->min_hit_score = 1;
    o->number_of_alignments = alignments;
    o->number_of_seeds = seeds;
    o->seg_enabled = 0;
    o->superfast = superfast;
}

static seq_t *make_query(const char *qint, int qlen) {
    seq_t *s = seq_alloc();
    seq_id(s, "q", 1);
    seq_seq(s, (char *)qint, qlen, 0);
    return s;
}

/* ------------------------------------------------------------- seeds */

/* For every query position i in [0, qlen - min_hit_length): lower bound
 * (or -2 when the position is skipped by _bad_prefix), and sa_hsp at pos and
 * pos-1 exactly as query_find_suffixes evaluates them (src/query.c:104-131).
 * hsp_len_m1 is -3 when pos == 0 (not evaluated). */
void ref_seed_list(void *dbh, const char *qint, int qlen, int min_hit_length,
                   const char *matrix, int64_t *pos, int32_t *hsp_score, int32_t *hsp_len,
                   int32_t *hsp_score_m1, int32_t *hsp_len_m1) {
    ref_db_t *r = (ref_db_t *)dbh;
    options_t o;
    set_options(&o, r, matrix, 100, 1e-3, 11, 1, 0.267, 0.041, 0.14, min_hit_length, 300000, 5000, 1);
    seq_t *q = make_query(qint, qlen);
    int n = qlen - min_hit_length;
    for (int i = 0; i < n; ++i) {
        saidx64_t p = -1, nm, lp;
        hsp_score[i] = hsp_len[i] = hsp_score_m1[i] = hsp_len_m1[i] = -3;
        if (upper_aa_only(seq_ptr(q)[i]) == 'V') { pos[i] = -2; continue; }
        sa_search(&r->db, q, i, 0, &p, &nm, &lp);
        pos[i] = p;
        int gs = 0, gl = 0;
        sa_hsp(&r->db, q, i, p, &o, &gs, &gl);
        hsp_score[i] = gs; hsp_len[i] = gl;
        if (p != 0) {
            gs = 0; gl = 0;
            sa_hsp(&r->db, q, i, p - 1, &o, &gs, &gl);
            hsp_score_m1[i] = gs; hsp_len_m1[i] = gl;
        }
    }
    seq_free(q);
}

/* One sa_search call (src/search.c:237-362) with all three outputs; returns
 * its return value. */
int ref_sa_search(void *dbh, const char *qint, int qlen, int64_t offset, int64_t length,
                  int64_t *idx, int64_t *num_matches, int64_t *last_position) {
    ref_db_t *r = (ref_db_t *)dbh;
    seq_t *q = make_query(qint, qlen);
    saidx64_t p = -7, nm = -7, lp = -7;
    int rc = sa_search(&r->db, q, offset, length, &p, &nm, &lp);
    *idx = p; *num_matches = nm; *last_position = lp;
    seq_free(q);
    return rc;
}

/* One sa_hsp call (src/search.c:99-190) at SA row `row`, query offset off. */
void ref_hsp(void *dbh, const char *qint, int qlen, int off, int64_t row, const char *matrix,
             int32_t *score, int32_t *len) {
    ref_db_t *r = (ref_db_t *)dbh;
    options_t o;
    set_options(&o, r, matrix, 100, 1e-3, 11, 1, 0.267, 0.041, 0.14, 5, 300000, 5000, 1);
    seq_t *q = make_query(qint, qlen);
    int gs = 0, gl = 0;
    sa_hsp(&r->db, q, off, row, &o, &gs, &gl);
    *score = gs; *len = gl;
    seq_free(q);
}

/* ----------------------------------------------------- whole query run */

/* Per-hit record returned in hitlist traversal order (src/rbtree.c:653-669:
 * gapless score descending, newest first among equal scores). */
typedef struct {
    int64_t db_index;
    int32_t gapless_score, gapless_length, suffix_offset, is_aligned;
    int32_t rawscore, qstart, qend, sstart, send;
    int32_t length, mismatch, gapopen, pad;
    double identity, bitscore, evalue;
} ref_hit_t;

/* Runs one query through the reference state machine (src/engine.c:348-390)
 * with the pops of query_fetch_alignment_batch recorded.
 * pops: up to max_pops records of (row, offset, score, length, counted).
 * Returns the number of hits written to `hits` (capacity max_hits); the
 * number of pops performed is written to *npops and the number of counted
 * pops to *ncounted. */
int ref_query_run(void *dbh, const char *qint, int qlen, const char *matrix, int num_hits,
                  double evalue, int go, int ge, double lambda, double k, double H,
                  int min_hit_length, int seeds, int alignments, int superfast,
                  int64_t *pop_row, int32_t *pop_off, int32_t *pop_score, int32_t *pop_len,
                  int32_t *pop_counted, int64_t max_pops, int64_t *npops, int64_t *ncounted,
                  ref_hit_t *hits, int max_hits) {
    ref_db_t *r = (ref_db_t *)dbh;
    options_t o;
    set_options(&o, r, matrix, num_hits, evalue, go, ge, lambda, k, H, min_hit_length, seeds,
                alignments, superfast);
    seq_t *qs = make_query(qint, qlen);
    query_t *q = query_alloc(qs, &r->db, &o);

    query_find_suffixes(q);

    /* the loop of query_fetch_alignment_batch (src/query.c:151-157), with
     * every pop recorded */
    saidx64_t SAindex, Qoffset;
    int gs, gl, counter = 0;
    int64_t np = 0;
    hit_t *h;
    while (pqueue_next(q->pq, &SAindex, &Qoffset, &gs, &gl) == 0) {
        h = hitlist_add(q->hl, q->db, SAindex, gs, gl, Qoffset);
        if (np < max_pops) {
            pop_row[np] = SAindex; pop_off[np] = (int32_t)Qoffset;
            pop_score[np] = gs; pop_len[np] = gl; pop_counted[np] = h != NULL;
        }
        np++;
        if (h != NULL) {
            if (++counter == o.number_of_seeds) break;
        }
    }
    *npops = np;
    *ncounted = counter;

    if (counter != 0) {
        query_perform_alignments(q);
        if (!o.superfast) query_perform_statistics(q);
    } else if (!o.superfast) {
        query_perform_statistics(q);
    }

    traversal_t *t = hitlist_traversal(q->hl);
    traversal_start(t);
    int nh = 0;
    while ((h = (hit_t *)traversal_next(t)) != NULL) {
        if (nh < max_hits) {
            ref_hit_t *o2 = &hits[nh];
            o2->db_index = (int64_t)h->db_index;
            o2->gapless_score = h->gapless_score;
            o2->gapless_length = h->gapless_length;
            o2->suffix_offset = h->suffix_offset;
            o2->is_aligned = h->is_aligned;
            o2->rawscore = h->rawscore;
            o2->qstart = h->qstart; o2->qend = h->qend;
            o2->sstart = h->sstart; o2->send = h->send;
            o2->length = h->length; o2->mismatch = h->mismatch; o2->gapopen = h->gapopen;
            o2->pad = 0;
            o2->identity = h->identity; o2->bitscore = h->bitscore; o2->evalue = h->evalue;
        }
        nh++;
    }
    traversal_free(t);
    query_free(q);  /* frees qs */
    return nh;
}

/* ----------------------------------------------------------------- SEG */

static int seg_ready = 0;

/* run_seg on an upper-cased residue string, in place (src/seg_wrapper.c:15-49). */
void ref_seg(char *residues, int len) {
    if (!seg_ready) { initialise_seg(); seg_ready = 1; }
    seq_t *s = seq_alloc();
    seq_id(s, "s", 1);
    seq_seq(s, residues, len, 0);
    run_seg(s);
    memcpy(residues, seq_ptr(s), len);
    seq_free(s);
}
