/*
 * tpzh_stats.c -- the --blasttab columns of one printed hit, with the
 * results of ssw_align_stats (src/ssw.c:900-978):
 *
 * 1. start coordinates: a reverse local-alignment pass over the subject
 *    columns ref_end1 .. 0 against the query prefix read[0..read_end1]
 *    reversed, computed with the striped SSW recurrence of the forward pass
 *    (u8 lane length ceil(n/16) when bias + score1 < 255, else i16 length
 *    ceil(n/8), src/ssw.c:929-935), stopping at the first column whose
 *    maximum equals score1 (the `terminate` test, :285/:488) -- the padded
 *    striped rows (score 0) take part in that column maximum;
 * 2. length / mismatches / gap opens / identity: banded Gotoh with the band
 *    doubled until its maximum reaches score1 and the traceback rules of
 *    banded_sw (src/ssw.c:538-784), including that the walk stops when the
 *    row index reaches 0 and compares residues after each move.
 */
#include "tpzh.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>

#define MAX2(a, b) ((a) > (b) ? (a) : (b))

/* reverse pass: returns the column (original subject index) where the
 * maximum was reached and the row in reversed-query coordinates */
static void reverse_pass(const int8_t *qrev, int32_t qlen, const int8_t *ref, int32_t ncol,
                         const int8_t *mat, int go, int ge, int word, int bias, int terminate,
                         int32_t *end_ref, int32_t *end_read) {
    const int lanes = word ? 8 : 16;
    const int seg = qlen > 0 ? (qlen + lanes - 1) / lanes : 0;
    const int rows = seg * lanes;                     /* striped slots incl. padding */
    int32_t *E = calloc(rows + 1, sizeof(int32_t));
    int32_t *Hp = calloc(rows + 1, sizeof(int32_t));
    int32_t *Hc = calloc(rows + 1, sizeof(int32_t));
    int32_t best = 0, bc = word ? 0 : -1, br = 0;
    for (int32_t c = ncol - 1; c >= 0; --c) {
        const int8_t *mrow = mat + 25 * ref[c];
        int32_t F = 0, Fm = 0, colmax = 0;
        int32_t cbest = 0, crow = 0;
        for (int32_t r = 0; r < rows; ++r) {
            if (r % seg == 0) Fm = 0;
            const int32_t D = r ? Hp[r - 1] : 0;
            const int32_t sc = r < qlen ? mrow[qrev[r]] : 0;
            int32_t hp = MAX2(0, D + sc);
            hp = MAX2(hp, E[r]);
            hp = MAX2(hp, Fm);
            const int32_t h = MAX2(hp, F);
            E[r] = MAX2(0, MAX2(E[r] - ge, hp - go));
            Fm = MAX2(0, MAX2(Fm - ge, hp - go));
            F = MAX2(0, MAX2(F - ge, h - go));
            Hc[r] = h;
            if (h > colmax) colmax = h;
            if (r < qlen && h > cbest) { cbest = h; crow = r; }
        }
        int32_t *t = Hp; Hp = Hc; Hc = t;
        if (cbest > best) {
            best = cbest;
            if ((!word && best + bias >= 255) || (word && best >= 32767)) break;
            bc = c;
            br = crow;
        }
        if (colmax == terminate) break;
    }
    free(E); free(Hp); free(Hc);
    *end_ref = bc;
    *end_read = best > 0 ? br : 0;
}

/* banded_sw: band doubling from band_width until the maximum reaches score,
 * then traceback from the bottom-right cell */
static int banded(const int8_t *ref, const int8_t *read, int32_t refLen, int32_t readLen,
                  int32_t score, int go, int ge, int32_t band, const int8_t *mat,
                  int32_t *length, int32_t *gapopen, int32_t *mismatch, double *identity) {
    *length = 0; *gapopen = 0; *mismatch = 0; *identity = 0.0;
    int32_t max = 0;
    int64_t s2 = 1024;
    int8_t *dir = NULL;
    int32_t width = 0, width_d = 0;
    int32_t *h_b = NULL, *e_b = NULL, *h_c = NULL;
    int32_t cap = 0;
    do {
        width = band * 2 + 3;
        width_d = band * 2 + 1;
        if (width + 1 > cap) {
            cap = width + 1;
            h_b = realloc(h_b, sizeof(int32_t) * cap);
            e_b = realloc(e_b, sizeof(int32_t) * cap);
            h_c = realloc(h_c, sizeof(int32_t) * cap);
            memset(h_b, 0, sizeof(int32_t) * cap);
            memset(e_b, 0, sizeof(int32_t) * cap);
            memset(h_c, 0, sizeof(int32_t) * cap);
        }
        int64_t need = (int64_t)width_d * readLen * 3;
        if (need > INT_MAX) goto too_big;
        while (need >= s2) {
            /* next power of two above s2 */
            int64_t x = s2;
            x |= x >> 1; x |= x >> 2; x |= x >> 4; x |= x >> 8; x |= x >> 16; x |= x >> 32;
            s2 = x + 1;
            if (s2 >= INT_MAX) goto too_big;
        }
        dir = realloc(dir, (size_t)s2);
        for (int32_t j = 1; j < width - 1; ++j) h_b[j] = 0;
        for (int32_t i = 0; i < readLen; ++i) {
            int32_t beg = i - band > 0 ? i - band : 0;
            int32_t end = i + band < refLen - 1 ? i + band : refLen - 1;
            const int32_t edge = end + 1 < width - 1 ? end + 1 : width - 1;
            int32_t f = 0, u = 0;
            h_b[0] = e_b[0] = h_b[edge] = e_b[edge] = h_c[0] = 0;
            int8_t *dl = dir + (int64_t)width_d * i * 3;
            const int32_t xi = i - band > 0 ? i - band : 0;          /* row i */
            const int32_t xp = i - 1 - band > 0 ? i - 1 - band : 0;  /* row i-1 */
            for (int32_t j = beg; j <= end; ++j) {
                u = j - xi + 1;
                const int32_t e = j - xp + 1, b = j - 1 - xi + 1, d = j - 1 - xp + 1;
                const int32_t de = (j - xi) * 3, df = de + 1, dh = de + 2;
                int32_t t1 = i == 0 ? -go : h_b[e] - go;
                int32_t t2 = i == 0 ? -ge : e_b[e] - ge;
                e_b[u] = t1 > t2 ? t1 : t2;
                dl[de] = t1 > t2 ? 3 : 2;
                t1 = h_c[b] - go;
                t2 = f - ge;
                f = t1 > t2 ? t1 : t2;
                dl[df] = t1 > t2 ? 5 : 4;
                const int32_t e1 = e_b[u] > 0 ? e_b[u] : 0, f1 = f > 0 ? f : 0;
                t1 = e1 > f1 ? e1 : f1;
                t2 = h_b[d] + mat[ref[j] * 25 + read[i]];
                h_c[u] = t1 > t2 ? t1 : t2;
                if (h_c[u] > max) max = h_c[u];
                if (t1 <= t2) dl[dh] = 1;
                else dl[dh] = e1 > f1 ? dl[de] : dl[df];
            }
            for (int32_t j = 1; j <= u; ++j) h_b[j] = h_c[j];
        }
        band *= 2;
    } while (max < score);
    band /= 2;

    {
        int32_t i = readLen - 1, j = refLen - 1, identical = 0, m = 2;
        char op = 'M', prev = 'M';
        int8_t *dl = dir + (int64_t)width_d * i * 3;
        while (i > 0) {
            const int32_t x = (i - band > 0 ? i - band : 0);
            const int64_t at = (int64_t)(j - x) * 3 + m;
            if (at < 0 || at >= (int64_t)width_d * 3) break;   /* outside the band */
            switch (dl[at]) {
            case 1: --i; --j; m = 2; dl -= width_d * 3; op = 'M'; break;
            case 2: --i; m = 0; dl -= width_d * 3; op = 'I'; break;
            case 3: --i; m = 2; dl -= width_d * 3; op = 'I'; break;
            case 4: --j; m = 1; op = 'D'; break;
            case 5: --j; m = 2; op = 'D'; break;
            default:
                free(dir); free(h_b); free(e_b); free(h_c);
                return 0;
            }
            if (op == 'M') {
                if (read[i] != ref[j]) (*mismatch)++;
                else identical++;
            }
            if ((op == 'I' && prev != 'I') || (op == 'D' && prev != 'D')) (*gapopen)++;
            (*length)++;
            prev = op;
        }
        *identity = identical / (double)*length;
    }
    free(dir); free(h_b); free(e_b); free(h_c);
    return 1;

too_big:
    *length = *gapopen = *mismatch = -1;
    *identity = -1.0;
    free(dir); free(h_b); free(e_b); free(h_c);
    return 0;
}

int tpzh_align_stats(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                     const int8_t *mat625, int gap_open, int gap_extend, int32_t read_end1,
                     int32_t ref_end1, int32_t score1, tpzh_stats *out) {
    (void)qlen; (void)slen;
    int bias = 0;
    for (int i = 0; i < 625; ++i) if (mat625[i] < bias) bias = mat625[i];
    bias = -bias;
    const int32_t n = read_end1 + 1;
    if (n <= 0 || ref_end1 < 0) {
        out->qstart = out->sstart = out->length = out->gapopen = out->mismatch = -1;
        out->identity = -1.0;
        return 0;
    }
    int8_t *rev = malloc(n);
    for (int32_t i = 0; i < n; ++i) rev[i] = q[read_end1 - i];
    const int word = !((bias + score1) < 255);
    int32_t rref, rread;
    reverse_pass(rev, n, s, ref_end1 + 1, mat625, gap_open, gap_extend, word, bias,
                 word ? (score1 & 0xFFFF) : (score1 & 0xFF), &rref, &rread);
    free(rev);
    out->sstart = rref;
    out->qstart = read_end1 - rread;
    if (rref < 0) {
        out->length = out->gapopen = out->mismatch = -1;
        out->identity = -1.0;
        return 0;
    }
    const int32_t refLen = ref_end1 - rref + 1;
    const int32_t readLen = read_end1 - out->qstart + 1;
    const int32_t bw = abs(refLen - readLen) + 1;
    return banded(s + rref, q + out->qstart, refLen, readLen, score1, gap_open, gap_extend, bw,
                  mat625, &out->length, &out->gapopen, &out->mismatch, &out->identity);
}
