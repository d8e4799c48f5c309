/*
 * oracle.c -- CPU restatement of the TOPAZ search hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Only tests/, the smoke check and
 * the cpu_baseline leg of bench.py load it; the product never does.  It is
 * pinned against the unmodified reference compiled into oracle/_ref (see
 * tests/test_oracle_pin.py) and against committed golden vectors
 * (tests/golden/).
 *
 * Plain scalar C, written for clarity rather than speed.  Each function cites
 * the reference lines whose behaviour it restates (paths inside the TOPAZ
 * source tree).
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define MAX2(a, b) ((a) > (b) ? (a) : (b))
#define MIN2(a, b) ((a) < (b) ? (a) : (b))

/* ====================================================================== */
/* Smith-Waterman                                                          */
/* ====================================================================== */

/*
 * Striped SSW computes local affine alignment in 16 (u8) or 8 (i16) lanes of
 * segLen = ceil(qlen/lanes) query rows each (src/ssw.c:93-118, :334-356).
 * Its result equals the following recurrence over query rows r and subject
 * columns c, where "lane start" means r % segLen == 0:
 *
 *   Hp(r,c) = max(0, H(r-1,c-1) + M[s_c][q_r], E(r,c), Fm(r,c))
 *             -- main loop, src/ssw.c:203-228 / :428-452
 *   H(r,c)  = max(Hp(r,c), F(r,c))
 *             -- after the lazy-F loop, src/ssw.c:232-262 / :455-466
 *   E(r,c+1)= max(E(r,c) - ge, Hp(r,c) - go)        (from the main-loop H)
 *   Fm(r+1) = lane start ? 0 : max(Fm(r) - ge, Hp(r) - go)   (in-lane F)
 *   F(r+1)  = max(F(r) - ge, H(r) - go)             (F across lanes too)
 *
 * with all of E, F, Fm floored at 0 (saturating subtraction).  E is fed from
 * the main-loop H, so a vertical gap that crossed a lane boundary cannot turn
 * into a horizontal gap in the next column; that is the one place where SSW
 * differs from textbook Gotoh, and why the lane length matters.
 *
 * Result (src/ssw.c:264-297, :469-500): the maximum H; ref_end = the first
 * column in which that maximum appears (the max only moves on a strict
 * increase); read_end = the smallest row holding the maximum in that column.
 */
static int sw_lane_model(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                         const int8_t *mat, int go, int ge, int32_t seg_len, int gotoh,
                         int32_t *ref_end, int32_t *read_end) {
    int32_t *E = calloc(qlen + 1, sizeof(int32_t));
    int32_t *Hprev = calloc(qlen + 1, sizeof(int32_t));
    int32_t *Hcur = calloc(qlen + 1, sizeof(int32_t));
    int32_t best = 0, bc = -1, br = qlen - 1;
    for (int32_t c = 0; c < slen; ++c) {
        const int8_t *mrow = mat + 25 * s[c];
        int32_t F = 0, Fm = 0;
        for (int32_t r = 0; r < qlen; ++r) {
            if (!gotoh && r % seg_len == 0) Fm = 0;
            int32_t D = r ? Hprev[r - 1] : 0;
            int32_t hp = MAX2(0, D + mrow[q[r]]);
            hp = MAX2(hp, E[r]);
            if (!gotoh) hp = MAX2(hp, Fm);
            int32_t h = MAX2(hp, F);
            int32_t ebase = gotoh ? h : hp;
            E[r] = MAX2(0, MAX2(E[r] - ge, ebase - go));
            if (!gotoh) Fm = MAX2(0, MAX2(Fm - ge, hp - go));
            F = MAX2(0, MAX2(F - ge, h - go));
            Hcur[r] = h;
            if (h > best) { best = h; bc = c; br = r; }
        }
        int32_t *t = Hprev; Hprev = Hcur; Hcur = t;
    }
    free(E); free(Hprev); free(Hcur);
    *ref_end = bc;
    /* With no positive cell the end-row scan (src/ssw.c:289-297) matches the
     * never-written all-zero column at its first slot: row 0. */
    *read_end = best > 0 ? br : 0;
    return best;
}

static int mat_bias(const int8_t *mat) {
    /* ssw_init: bias = |min(0, min over the n*n table)| (src/ssw.c:805-812) */
    int b = 0;
    for (int i = 0; i < 625; ++i) if (mat[i] < b) b = mat[i];
    return -b;
}

/* ssw_align with score_size 2 (src/ssw.c:835-897): the u8 pass; if it
 * saturates (max + bias >= 255) the i16 pass; if that reaches 32767 the
 * alignment is dropped (returns 1).  Valid for gap_open > gap_extend, the
 * case in which the i16 lazy-F early exit (src/ssw.c:464) is exact. */
int orc_ssw_align(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                  const int8_t *mat25, int gap_open, int gap_extend,
                  int32_t *score, int32_t *ref_end, int32_t *read_end) {
    int bias = mat_bias(mat25);
    int32_t re, rd;
    int32_t m = sw_lane_model(q, qlen, s, slen, mat25, gap_open, gap_extend, (qlen + 15) / 16, 0,
                              &re, &rd);
    if (m + bias >= 255) {
        m = sw_lane_model(q, qlen, s, slen, mat25, gap_open, gap_extend, (qlen + 7) / 8, 0, &re,
                          &rd);
        if (m >= 32767) {
            *score = 32767; *ref_end = -1; *read_end = -1;
            return 1;
        }
    }
    *score = m; *ref_end = re; *read_end = rd;
    return 0;
}

int orc_gotoh_align(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                    const int8_t *mat25, int gap_open, int gap_extend,
                    int32_t *score, int32_t *ref_end, int32_t *read_end) {
    *score = sw_lane_model(q, qlen, s, slen, mat25, gap_open, gap_extend, 1, 1, ref_end, read_end);
    return 0;
}

typedef struct {
    int64_t n, t, nt;
    const int8_t *q; const int64_t *qoff; const int32_t *qlen;
    const int8_t *s; const int64_t *soff; const int32_t *slen;
    const int8_t *mat; int go, ge;
    int32_t *score, *ref_end, *read_end, *status;
} orc_batch_t;

static void *orc_batch_worker(void *v) {
    orc_batch_t *b = v;
    for (int64_t i = b->t; i < b->n; i += b->nt)
        b->status[i] = orc_ssw_align(b->q + b->qoff[i], b->qlen[i], b->s + b->soff[i], b->slen[i],
                                     b->mat, b->go, b->ge, &b->score[i], &b->ref_end[i],
                                     &b->read_end[i]);
    return NULL;
}

void orc_ssw_batch(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                   const int8_t *s, const int64_t *soff, const int32_t *slen,
                   const int8_t *mat25, int go, int ge, int nthreads,
                   int32_t *score, int32_t *ref_end, int32_t *read_end, int32_t *status) {
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = malloc(sizeof(pthread_t) * nthreads);
    orc_batch_t *a = malloc(sizeof(orc_batch_t) * nthreads);
    for (int t = 0; t < nthreads; ++t) {
        orc_batch_t b = {n, t, nthreads, q, qoff, qlen, s, soff, slen, mat25, go, ge,
                         score, ref_end, read_end, status};
        a[t] = b;
        pthread_create(&th[t], NULL, orc_batch_worker, &a[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th); free(a);
}

/* ====================================================================== */
/* Alphabet                                                                */
/* ====================================================================== */

/* Internal alphabet letter -> matrix index (aa_table2, src/lexicographical.h
 * :19-33).  The internal letters 'A'..'Y' stand for the amino acids
 * "ACMLJIVTSKRQZEDBNHYFWXP*G" in that order (src/lexicographical.h:135-160);
 * every other byte maps to X (23). */
static int aa_index_of_internal(int c) {
    static const char internal_to_aa[] = "ACMLJIVTSKRQZEDBNHYFWXP*G";
    static const char matrix_order[] = "ARNDCQEGHILKMFPSTWYVBJZX*";
    if (c >= 'a' && c <= 'y') c -= 32;
    if (c < 'A' || c > 'Y') return 23;
    char aa = internal_to_aa[c - 'A'];
    const char *p = strchr(matrix_order, aa);
    return (int)(p - matrix_order);
}

/* upper_aa_only (src/lexicographical.h:60-75): 'A'..'Y', '*', '\n' pass,
 * everything else reads as 'V' (internal X). */
static int upper_aa_only(int c) {
    if ((c >= 'A' && c <= 'Y') || c == '*' || c == '\n') return c;
    return 'V';
}

/* ====================================================================== */
/* Seeding                                                                 */
/* ====================================================================== */

/* Sign of (T suffix at t) - P as _compare decides it (src/search.c:18-30):
 * byte-wise; a text suffix that ends first is smaller; P being a prefix of
 * the suffix counts as equal. */
static int suffix_cmp(const char *T, int64_t Tsize, int64_t t, const char *P, int64_t Psize) {
    int64_t i = t, j = 0;
    while (i < Tsize && j < Psize) {
        int r = (int)T[i] - (int)P[j];
        if (r) return r;
        ++i; ++j;
    }
    return j == Psize ? 0 : -1;
}

/* sa_search's idx (src/search.c:237-362) is the lower bound of P: the number
 * of suffixes strictly smaller than P (the first row whose suffix has P as a
 * prefix when there is one). */
int64_t orc_lower_bound(const char *T, int64_t Tsize, const int64_t *SA,
                        const char *P, int64_t Psize) {
    int64_t lo = 0, hi = Tsize;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (suffix_cmp(T, Tsize, SA[mid], P, Psize) < 0) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* sa_hsp (src/search.c:99-190) for a text position idx = SA[row]. */
static void hsp_at(const char *T, int64_t Tsize, int64_t idx, const char *Q, int32_t qlen,
                   int32_t off, const int8_t *mat, int32_t *score, int32_t *len) {
    const char *t = T + idx;
    const char *qq = Q + off;
    if (t[0] != qq[0]) { *len = -1; return; }     /* :113-116, score untouched */
    int64_t mr = MIN2(Tsize - idx, (int64_t)(qlen - off));
    mr = MIN2(mr, 128);                              /* :119 */
    int32_t run = 0, best_r = 0, arg_r = 0;
    for (int64_t i = 0; i < mr; ++i) {               /* :126-149 */
        if (t[i] == '\n') break;
        run += mat[aa_index_of_internal(t[i]) * 25 + aa_index_of_internal(upper_aa_only(qq[i]))];
        if (run >= best_r) { best_r = run; arg_r = (int32_t)i; }
    }
    int64_t ml = MIN2(idx, (int64_t)off);
    ml = MIN2(ml, 128);                              /* :158 */
    int32_t best_l = 0, arg_l = 0;
    run = 0;
    for (int64_t i = 1; i < ml; ++i) {               /* :161-183 */
        if (t[-i] == '\n') break;
        run += mat[aa_index_of_internal(t[-i]) * 25 + aa_index_of_internal(upper_aa_only(qq[-i]))];
        if (run >= best_l) { best_l = run; arg_l = (int32_t)i; }
    }
    *score = best_l + best_r;                        /* :186-187 */
    *len = arg_l + arg_r;
}

void orc_hsp(const char *T, int64_t Tsize, const int64_t *SA, const char *Q, int32_t qlen,
             int32_t off, int64_t row, const int8_t *mat25, int32_t *score, int32_t *len) {
    hsp_at(T, Tsize, SA[row], Q, qlen, off, mat25, score, len);
}

/* ====================================================================== */
/* One query                                                               */
/* ====================================================================== */

/* Both ordered containers of the reference are red-black trees in which an
 * equal key goes right (src/rbtree.c:70-78), so each behaves as a list sorted
 * by key with equal keys in insertion order: the max end pops the newest of
 * the largest key (rb_popmax, :410-427), the min end the oldest of the
 * smallest (rb_popmin/rb_getmin, :429-457), rb_reput re-inserts as newest
 * (:496-505) and traversal visits keys descending, newest first (:653-669).
 * The restatement keys every entry by (score, insertion stamp) in plain
 * binary heaps, which orders them identically. */

typedef struct { int64_t row; int32_t off, dir, score, len; int64_t stamp; } cursor_t;

static int cur_gt(const cursor_t *a, const cursor_t *b) {
    return a->score != b->score ? a->score > b->score : a->stamp > b->stamp;
}

typedef struct { cursor_t *v; int64_t n, cap; } maxheap_t;

static void mh_push(maxheap_t *h, cursor_t c) {
    if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 256; h->v = realloc(h->v, h->cap * sizeof(cursor_t)); }
    int64_t i = h->n++;
    h->v[i] = c;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (!cur_gt(&h->v[i], &h->v[p])) break;
        cursor_t t = h->v[i]; h->v[i] = h->v[p]; h->v[p] = t; i = p;
    }
}

static cursor_t mh_pop(maxheap_t *h) {
    cursor_t top = h->v[0];
    h->v[0] = h->v[--h->n];
    int64_t i = 0;
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < h->n && cur_gt(&h->v[l], &h->v[m])) m = l;
        if (r < h->n && cur_gt(&h->v[r], &h->v[m])) m = r;
        if (m == i) break;
        cursor_t t = h->v[i]; h->v[i] = h->v[m]; h->v[m] = t; i = m;
    }
    return top;
}

typedef struct {
    int64_t protein;
    int32_t score, len, off;
    int64_t stamp;
    int64_t heap_pos;
} hitrec_t;

/* min-heap of hit indices ordered by (score asc, stamp asc), with positions */
typedef struct { int32_t *v; int64_t n; hitrec_t *recs; } minheap_t;

static int hit_lt(const hitrec_t *a, const hitrec_t *b) {
    return a->score != b->score ? a->score < b->score : a->stamp < b->stamp;
}

static void hh_swap(minheap_t *h, int64_t i, int64_t j) {
    int32_t t = h->v[i]; h->v[i] = h->v[j]; h->v[j] = t;
    h->recs[h->v[i]].heap_pos = i;
    h->recs[h->v[j]].heap_pos = j;
}

static void hh_up(minheap_t *h, int64_t i) {
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (!hit_lt(&h->recs[h->v[i]], &h->recs[h->v[p]])) break;
        hh_swap(h, i, p); i = p;
    }
}

static void hh_down(minheap_t *h, int64_t i) {
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < h->n && hit_lt(&h->recs[h->v[l]], &h->recs[h->v[m]])) m = l;
        if (r < h->n && hit_lt(&h->recs[h->v[r]], &h->recs[h->v[m]])) m = r;
        if (m == i) break;
        hh_swap(h, i, m); i = m;
    }
}

/* db_index (src/db.c:176-205): protein whose [start, start+len] (delimiter
 * included) holds text position pos. */
static int64_t protein_of(const int64_t *pstart, int64_t Psize, int64_t pos) {
    int64_t lo = 0, hi = Psize - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) / 2;
        if (pstart[mid] <= pos) lo = mid; else hi = mid - 1;
    }
    return lo;
}

static int hit_desc_cmp(const void *a, const void *b) {
    const hitrec_t *x = a, *y = b;
    if (x->score != y->score) return x->score > y->score ? -1 : 1;
    return x->stamp > y->stamp ? -1 : (x->stamp < y->stamp ? 1 : 0);
}

int orc_query_run(const char *T, int64_t Tsize, const int64_t *SA, const int64_t *pstart,
                  int64_t Psize, const char *qint, int32_t qlen, const int8_t *mat25,
                  const orc_opts_t *o, int64_t *pop_row, int32_t *pop_off, int32_t *pop_score,
                  int32_t *pop_len, int32_t *pop_counted, int64_t max_pops, int64_t *npops,
                  int64_t *ncounted, orc_hit_t *hits, int32_t max_hits) {
    /* SA entries past Tsize read the zero fill of the mapped file's last page
     * (src/db.c:362 maps .SA; search.c:100 and hit.c:138 index it with rows
     * up to 8*Tsize, db.c:249-251).  Beyond that page the reference faults. */
    int64_t sa_limit = ((Tsize * 8 + 4095) / 4096) * 4096 / 8;
    int fault = 0;
#define SA_AT(row) ((row) < Tsize ? SA[row] : ((row) < sa_limit ? 0 : (fault = 1, 0)))

    int64_t stamp = 0;
    maxheap_t pq = {0};
    int minlen = o->min_hit_length;

    /* query_find_suffixes (src/query.c:94-137) */
    for (int32_t i = 0; i < qlen - minlen; ++i) {
        if (upper_aa_only(qint[i]) == 'V') continue;     /* _bad_prefix :88-92 */
        int64_t pos = orc_lower_bound(T, Tsize, SA, qint + i, qlen - i);
        int32_t sc = 0, ln = 0;
        int64_t idx = SA_AT(pos);
        if (fault) goto faulted;
        hsp_at(T, Tsize, idx, qint, qlen, i, mat25, &sc, &ln);
        if (ln >= minlen) { cursor_t c = {pos, i, 1, sc, ln, stamp++}; mh_push(&pq, c); }
        if (pos != 0) {
            sc = 0; ln = 0;
            hsp_at(T, Tsize, SA[pos - 1], qint, qlen, i, mat25, &sc, &ln);
            if (ln >= minlen) { cursor_t c = {pos - 1, i, -1, sc, ln, stamp++}; mh_push(&pq, c); }
        }
    }

    /* hitlist_alloc capacity (src/hit.c:106-109) */
    int64_t cap = o->alignments;
    if (qlen > 3000) cap = (int64_t)(1.5 * o->num_hits);

    hitrec_t *recs = malloc(sizeof(hitrec_t) * (cap + 2));
    int32_t *free_ids = malloc(sizeof(int32_t) * (cap + 2));
    int64_t nfree = cap + 2;
    for (int64_t i = 0; i < nfree; ++i) free_ids[i] = (int32_t)(nfree - 1 - i);
    minheap_t hh = {malloc(sizeof(int32_t) * (cap + 2)), 0, recs};
    int32_t *hit_of = malloc(sizeof(int32_t) * Psize);
    for (int64_t p = 0; p < Psize; ++p) hit_of[p] = -1;

    int64_t np = 0, counter = 0, hstamp = 0;
    /* query_fetch_alignment_batch loop (src/query.c:151-157) */
    while (pq.n > 0) {
        /* pqueue_next (src/priority_queue.c:36-56) */
        cursor_t c = mh_pop(&pq);
        int64_t row = c.row;
        int32_t gs = c.score, gl = c.len, off = c.off;
        c.row += c.dir;                                   /* suffix_increment */
        if (c.row >= 0 && c.row < Tsize * 8) {             /* db_valid_index */
            int64_t idx = SA_AT(c.row);
            if (fault) goto faulted2;
            hsp_at(T, Tsize, idx, qint, qlen, c.off, mat25, &c.score, &c.len);
            if (c.len >= minlen) { c.stamp = stamp++; mh_push(&pq, c); }
        }
        /* hitlist_add (src/hit.c:126-193) */
        int counted = 0;
        if (hh.n >= cap && recs[hh.v[0]].score >= gs) {
            counted = 1;
        } else {
            int64_t p = protein_of(pstart, Psize, SA_AT(row));
            if (fault) goto faulted2;
            int32_t h = hit_of[p];
            if (h < 0) {
                h = free_ids[--nfree];
                hitrec_t r = {p, gs, gl, off, hstamp++, hh.n};
                recs[h] = r;
                hit_of[p] = h;
                hh.v[hh.n++] = h;
                hh_up(&hh, hh.n - 1);
                if (hh.n > cap) {                            /* evict the worst */
                    int32_t w = hh.v[0];
                    hh_swap(&hh, 0, hh.n - 1);
                    hh.n--;
                    hh_down(&hh, 0);
                    hit_of[recs[w].protein] = -1;
                    free_ids[nfree++] = w;
                }
                counted = 1;
            } else if (recs[h].score < gs) {
                recs[h].score = gs; recs[h].len = gl; recs[h].stamp = hstamp++;
                hh_down(&hh, recs[h].heap_pos);
                hh_up(&hh, recs[h].heap_pos);
            }
        }
        if (np < max_pops) {
            pop_row[np] = row; pop_off[np] = off; pop_score[np] = gs; pop_len[np] = gl;
            pop_counted[np] = counted;
        }
        np++;
        if (counted && ++counter == o->seeds) break;
    }
    *npops = np;
    *ncounted = counter;

    /* hits in traversal order */
    int64_t nh = hh.n;
    hitrec_t *sorted = malloc(sizeof(hitrec_t) * (nh ? nh : 1));
    for (int64_t i = 0; i < nh; ++i) sorted[i] = recs[hh.v[i]];
    qsort(sorted, nh, sizeof(hitrec_t), hit_desc_cmp);

    /* query_perform_alignments (src/query.c:178-248) runs only when the
     * fetch counted something (:165-170) */
    int8_t *qidx = malloc(qlen > 0 ? qlen : 1);
    for (int32_t i = 0; i < qlen; ++i) qidx[i] = (int8_t)aa_index_of_internal(qint[i]);
    double db_size = (double)(uint64_t)(Tsize - Psize);
    /* align_using_ssw_profile constants (src/ssw_wrapper.c:179-181) */
    double correction = log(o->k * qlen * (uint64_t)(Tsize - Psize)) / o->H;
    double cq = fmax(qlen - correction, 1.0);
    double cdb = fmax(db_size - (correction * (uint64_t)Psize), 1.0);
    int8_t *sbuf = NULL;
    int64_t sbuf_cap = 0;
    for (int64_t i = 0; i < nh && i < max_hits; ++i) {
        orc_hit_t *out = &hits[i];
        hitrec_t *r = &sorted[i];
        out->db_index = r->protein;
        out->gapless_score = r->score;
        out->gapless_length = r->len;
        out->suffix_offset = r->off;
        out->is_aligned = 0;
        out->rawscore = -1; out->qend = -1; out->send = -1; out->status = 0;
        out->bitscore = INFINITY; out->evalue = INFINITY;
        if (counter == 0) continue;
        if (r->score < 40) {                              /* ssw_wrapper.c:171-176 */
            out->bitscore = 0; out->evalue = 1000; out->is_aligned = 1;
            continue;
        }
        int64_t st = pstart[r->protein];
        int64_t sl = 0;
        while (st + sl < Tsize && T[st + sl] != '\n') sl++;
        if (sl > sbuf_cap) { sbuf_cap = sl; sbuf = realloc(sbuf, sbuf_cap); }
        for (int64_t j = 0; j < sl; ++j) sbuf[j] = (int8_t)aa_index_of_internal(T[st + j]);
        int32_t sc, re, rd;
        int dropped = orc_ssw_align(qidx, qlen, sbuf, (int32_t)sl, mat25, o->gap_open,
                                    o->gap_extend, &sc, &re, &rd);
        if (dropped) { out->rawscore = 32767; out->status = 1; continue; }
        out->rawscore = sc; out->qend = rd; out->send = re;
        double bits = (o->lambda * sc - log(o->k));      /* :239-242 */
        double ev = cq * cdb * exp(-bits);
        ev = ev > 1.0e-180 ? ev : 0.0;
        out->bitscore = bits / M_LN2;
        out->evalue = ev;
        out->is_aligned = 1;
    }
    free(sbuf); free(qidx); free(sorted);
    free(recs); free(free_ids); free(hh.v); free(hit_of); free(pq.v);
    return (int)nh;

faulted2:
    free(recs); free(free_ids); free(hh.v); free(hit_of);
faulted:
    free(pq.v);
    return -1;
#undef SA_AT
}

/* output_top_hits (src/engine.c:193-248): aligned hits in traversal order,
 * stable sort by bitscore descending (glibc qsort is a stable merge sort
 * here; compare_bitscore src/utils.c:140-152), first num_hits, printed when
 * evalue <= threshold. */
int orc_rank_select(const orc_hit_t *hits, int32_t nhits, int32_t num_hits, double evalue,
                    int32_t *out_idx) {
    int32_t *idx = malloc(sizeof(int32_t) * (nhits ? nhits : 1));
    int32_t n = 0;
    for (int32_t i = 0; i < nhits; ++i) if (hits[i].is_aligned) idx[n++] = i;
    /* stable insertion sort on bitscore descending */
    for (int32_t i = 1; i < n; ++i) {
        int32_t v = idx[i], j = i - 1;
        while (j >= 0 && hits[idx[j]].bitscore < hits[v].bitscore) { idx[j + 1] = idx[j]; --j; }
        idx[j + 1] = v;
    }
    if (n > num_hits) n = num_hits;
    int32_t k = 0;
    for (int32_t i = 0; i < n; ++i) if (hits[idx[i]].evalue <= evalue) out_idx[k++] = idx[i];
    free(idx);
    return k;
}
