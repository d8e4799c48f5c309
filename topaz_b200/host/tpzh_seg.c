/*
 * tpzh_seg.c -- SEG low-complexity masking of query sequences.
 *
 * Restates the SEG algorithm (Wootton & Federhen, Comput. Chem. 17:149,
 * 1993) as TOPAZ runs it before seeding (run_seg, src/seg_wrapper.c:15-49:
 * window 12, trigger complexity 2.2, extension 2.5, maximal trim 100, hard
 * mask with 'X').  Every comparison is done on doubles computed in the same
 * order as src/seg/seg.c and src/seg/genwin.c so that the masks agree bit
 * for bit:
 *   - only the 20 standard residues ACDEFGHIKLMNPQRSTVWY (either case) are
 *     counted; other bytes are skipped (genwin.c:51-71);
 *   - a window's state is its multiset of non-zero residue counts kept in
 *     descending order; its entropy sums over that order (genwin.c:256-295);
 *   - segment trimming minimises log P(window) with ln n! taken from a table
 *     holding ln n! rounded to 6 decimals (src/seg/lnfac.h, reproduced here
 *     as the "%.6f" rendering of lgamma(n+1)), seg.c:292-408;
 *   - a segment found by extension is trimmed, a trigger window lost in the
 *     left trim is searched recursively, and neighbouring segments are merged
 *     by taking the next segment's end (seg.c:147-205, :412-451).
 */
#include "tpzh.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define SEG_WINDOW 12
#define SEG_LOCUT 2.2
#define SEG_HICUT 2.5
#define SEG_MAXTRIM 100
#define SEG_LN2 0.69314718055994530941723212145818
#define SEG_LN20 2.9957322735539909
#define SEG_DOWNSET ((SEG_WINDOW + 1) / 2 - 1)
#define SEG_UPSET (SEG_WINDOW - SEG_DOWNSET)

static int res_index[256];       /* residue -> 0..19, or -1 when not counted */
static double entropy_full[SEG_WINDOW + 1];
static double *lnfac_tab;
static int lnfac_n;
static int seg_ready;

static double lnfac(int n) {
    if (n < lnfac_n) return lnfac_tab[n];
    char buf[64];
    snprintf(buf, sizeof buf, "%.6f", lgamma((double)n + 1.0));
    return strtod(buf, NULL);
}

static void seg_init(void) {
    if (seg_ready) return;
    const char *aa = "ACDEFGHIKLMNPQRSTVWY";
    for (int i = 0; i < 256; ++i) res_index[i] = -1;
    for (int i = 0; aa[i]; ++i) {
        res_index[(unsigned char)aa[i]] = i;
        res_index[(unsigned char)(aa[i] + 32)] = i;
    }
    const double xw = SEG_WINDOW;
    for (int i = 1; i <= SEG_WINDOW; ++i) {
        const double x = i / xw;
        entropy_full[i] = -x * log(x) / SEG_LN2;
    }
    lnfac_n = 10001;
    lnfac_tab = malloc(sizeof(double) * lnfac_n);
    for (int n = 0; n < lnfac_n; ++n) {
        char buf[64];
        snprintf(buf, sizeof buf, "%.6f", lgamma((double)n + 1.0));
        lnfac_tab[n] = strtod(buf, NULL);
    }
    seg_ready = 1;
}

/* A window over s[start, start+len): residue counts and their descending
 * non-zero multiset (sv, zero-terminated, 21 slots). */
typedef struct {
    const char *s;
    int start, len, parent_len;
    int comp[20];
    int sv[21];
} window_t;

static void window_open(window_t *w, const char *s, int parent_len, int start, int len) {
    w->s = s; w->start = start; w->len = len; w->parent_len = parent_len;
    memset(w->comp, 0, sizeof w->comp);
    for (int i = start; i < start + len; ++i) {
        const int k = res_index[(unsigned char)s[i]];
        if (k >= 0) w->comp[k]++;
    }
    int n = 0;
    for (int k = 0; k < 20; ++k) if (w->comp[k]) w->sv[n++] = w->comp[k];
    for (int k = n; k < 21; ++k) w->sv[k] = 0;
    /* descending order */
    for (int a = 1; a < n; ++a) {
        int v = w->sv[a], b = a - 1;
        while (b >= 0 && w->sv[b] < v) { w->sv[b + 1] = w->sv[b]; --b; }
        w->sv[b + 1] = v;
    }
}

/* one class of count c shrinks by one: the last entry equal to c */
static void sv_dec(int *sv, int c) {
    int i = 0;
    while (sv[i] != 0) {
        if (sv[i] == c && sv[i + 1] < c) { sv[i] = c - 1; return; }
        ++i;
    }
}

/* one class of count c grows by one: the first entry equal to c (c = 0 is
 * the terminator slot) */
static void sv_inc(int *sv, int c) {
    int i = 0;
    while (sv[i] != c) ++i;
    sv[i]++;
}

/* move the window one residue right; 0 when it would leave its parent */
static int window_shift(window_t *w) {
    if (w->start + 1 + w->len > w->parent_len) return 0;
    const int out = res_index[(unsigned char)w->s[w->start]];
    const int in = res_index[(unsigned char)w->s[w->start + w->len]];
    w->start++;
    if (out >= 0) sv_dec(w->sv, w->comp[out]--);
    if (in >= 0) sv_inc(w->sv, w->comp[in]++);
    return 1;
}

static double sv_entropy(const int *sv) {
    int total = 0, n = 0;
    while (sv[n] != 0) total += sv[n++];
    double ent = 0.0;
    if (total == SEG_WINDOW) {
        for (int i = 0; i < n; ++i) ent += entropy_full[sv[i]];
        return ent;
    }
    if (total == 0) return 0.;
    const double rt = 1. / (double)total;
    for (int i = 0; i < n; ++i) {
        const double x = sv[i];
        ent += x * log(x * rt);
    }
    return -ent * rt / SEG_LN2;
}

/* ln of the number of ways to give the 20 residues the counts of sv */
static double sv_lnass(const int *sv) {
    double ans = lnfac(20);
    if (sv[0] == 0) return ans;
    int total = 20, cls = 1, prev = sv[0], i = 0;
    const int *p = sv;
    for (;;) {
        if (++i == 20) { ans -= lnfac(cls); break; }
        const int cur = *++p;
        if (cur == prev) { cls++; continue; }
        total -= cls;
        ans -= lnfac(cls);
        if (cur == 0) { ans -= lnfac(total); break; }
        cls = 1;
        prev = cur;
    }
    return ans;
}

static double sv_lnperm(const int *sv, int tot) {
    double ans = lnfac(tot);
    for (int i = 0; sv[i] != 0; ++i) ans -= lnfac(sv[i]);
    return ans;
}

static double sv_prob(const int *sv, int total) {
    const double totseq = ((double)total) * SEG_LN20;
    return sv_lnass(sv) + sv_lnperm(sv, total) - totseq;
}

typedef struct { int begin, end; } segment_t;
typedef struct { segment_t *v; int n, cap; } seglist_t;

static void seg_push(seglist_t *l, int b, int e) {
    if (l->n == l->cap) { l->cap = l->cap ? 2 * l->cap : 16; l->v = realloc(l->v, l->cap * sizeof(segment_t)); }
    l->v[l->n].begin = b; l->v[l->n].end = e; l->n++;
}

/* the most improbable sub-window of s[start, start+len) no shorter than
 * len - 100: adjusts [*left, *right] (absolute ends of that window) */
static void seg_trim(const char *s, int parent_len, int start, int len, int *left, int *right) {
    int lend = 0, rend = len - 1, minlen = 1;
    if (len - SEG_MAXTRIM > minlen) minlen = len - SEG_MAXTRIM;
    double minprob = 1.;
    for (int wl = len; wl > minlen; --wl) {
        window_t w;
        window_open(&w, s, start + len, start, wl);
        (void)parent_len;
        int i = 0;
        for (;;) {
            const double p = sv_prob(w.sv, wl);
            if (p < minprob) { minprob = p; lend = i; rend = wl + i - 1; }
            if (!window_shift(&w)) break;
            ++i;
        }
    }
    *left += lend;
    *right -= (len - rend - 1);
}

/* segseq on s[start, start+len) (a sub-window of the query); segments are
 * appended with absolute positions */
static void seg_search(const char *s, int start, int len, seglist_t *out) {
    if (SEG_WINDOW > len) return;
    double *H = malloc(sizeof(double) * len);
    for (int i = 0; i < len; ++i) H[i] = -1.;
    const int first = SEG_DOWNSET, last = len - SEG_UPSET;
    window_t w;
    window_open(&w, s, start + len, start, SEG_WINDOW);
    for (int i = first; i <= last; ++i) {
        H[i] = sv_entropy(w.sv);
        window_shift(&w);
    }
    int lowlim = first;
    for (int i = first; i <= last; ++i) {
        if (!(H[i] <= SEG_LOCUT && H[i] != -1)) continue;
        int j;
        for (j = i; j >= lowlim; --j) if (H[j] == -1 || H[j] > SEG_HICUT) break;
        const int loi = j + 1;
        for (j = i; j <= last; ++j) if (H[j] == -1 || H[j] > SEG_HICUT) break;
        const int hii = j - 1;
        int leftend = loi - SEG_DOWNSET;
        int rightend = hii + SEG_UPSET - 1;
        seg_trim(s, start + len, start + leftend, rightend - leftend + 1, &leftend, &rightend);
        if (i + SEG_UPSET - 1 < leftend) {
            /* the trigger window fell to the left trim: search the cut part */
            const int lend = loi - SEG_DOWNSET, rend = leftend - 1;
            seg_search(s, start + lend, rend - lend + 1, out);
        }
        seg_push(out, leftend + start, rightend + start);
        i = hii < rightend + SEG_DOWNSET ? hii : rightend + SEG_DOWNSET;
        lowlim = i + 1;
    }
    free(H);
}

int tpzh_seg_mask(char *seq, int len) {
    seg_init();
    seglist_t l = {0};
    seg_search(seq, 0, len, &l);
    if (l.n > 0) {
        /* mergesegs: an overlapping successor donates its end */
        int k = 0;
        for (int i = 1; i < l.n; ++i) {
            if (l.v[k].end >= l.v[i].begin) l.v[k].end = l.v[i].end;
            else l.v[++k] = l.v[i];
        }
        l.n = k + 1;
        for (int i = 0; i < l.n; ++i)
            if (l.v[i].end >= l.v[i].begin)
                memset(seq + l.v[i].begin, 'X', l.v[i].end - l.v[i].begin + 1);
    }
    const int n = l.n;
    free(l.v);
    return n;
}

/* The tables the device SEG uses (so that its doubles equal these):
 * ent_full[0..12] the full-window entropy terms, logxr[t * 13 + x] =
 * log(x * (1 / t)) for 1 <= x <= t <= 12 (the partial-window terms of
 * sv_entropy), lnfac[0..n) ln n! as rounded here. */
void tpzh_seg_tables(double *ent_full, double *logxr, double *lnfac_out, int n) {
    seg_init();
    for (int i = 0; i <= SEG_WINDOW; ++i) ent_full[i] = i ? entropy_full[i] : 0.0;
    for (int t = 0; t <= SEG_WINDOW; ++t)
        for (int x = 0; x <= SEG_WINDOW; ++x) {
            double v = 0.0;
            if (t >= 1 && x >= 1 && x <= t) {
                const double rt = 1. / (double)t;
                const double xd = x;
                v = log(xd * rt);
            }
            logxr[t * (SEG_WINDOW + 1) + x] = v;
        }
    for (int i = 0; i < n; ++i) lnfac_out[i] = lnfac(i);
}

