/*
 * tpzh_sais.c -- suffix array construction by induced sorting (SA-IS;
 * Nong, Zhang & Chan, "Two efficient algorithms for linear time suffix
 * array construction", IEEE Trans. Comput. 60:1471, 2011).
 *
 * The suffix array of a text is unique, so this produces the same .SA
 * bytes as the divsufsort64 call of `topaz index` (src/index.c:65-69):
 * suffixes in byte order, a suffix that is a prefix of another first.
 */
#include "tpzh.h"

#include <stdlib.h>
#include <string.h>

typedef int64_t idx_t;

/* L/S types: 1 = S.  isLMS(i): S-type with an L-type left neighbour */
#define IS_LMS(t, i) ((i) > 0 && (t)[i] && !(t)[(i) - 1])

static void bucket_bounds(const idx_t *s, idx_t n, idx_t K, idx_t *bkt, int ends) {
    memset(bkt, 0, sizeof(idx_t) * K);
    for (idx_t i = 0; i < n; ++i) bkt[s[i]]++;
    idx_t sum = 0;
    for (idx_t c = 0; c < K; ++c) {
        sum += bkt[c];
        bkt[c] = ends ? sum : sum - bkt[c];
    }
}

static void induce(const idx_t *s, const uint8_t *t, idx_t *SA, idx_t n, idx_t K, idx_t *bkt) {
    bucket_bounds(s, n, K, bkt, 0);
    for (idx_t i = 0; i < n; ++i) {
        const idx_t j = SA[i] - 1;
        if (SA[i] > 0 && !t[j]) SA[bkt[s[j]]++] = j;
    }
    bucket_bounds(s, n, K, bkt, 1);
    for (idx_t i = n - 1; i >= 0; --i) {
        const idx_t j = SA[i] - 1;
        if (SA[i] > 0 && t[j]) SA[--bkt[s[j]]] = j;
    }
}

/* s[n-1] must be the unique smallest symbol 0; symbols < K */
static int sais(idx_t *s, idx_t n, idx_t K, idx_t *SA) {
    uint8_t *t = malloc(n);
    idx_t *bkt = malloc(sizeof(idx_t) * K);
    if (!t || !bkt) { free(t); free(bkt); return -1; }
    t[n - 1] = 1;
    for (idx_t i = n - 2; i >= 0; --i)
        t[i] = s[i] < s[i + 1] || (s[i] == s[i + 1] && t[i + 1]);

    /* stage 1: LMS suffixes at their bucket ends, induce, sort LMS substrings */
    bucket_bounds(s, n, K, bkt, 1);
    for (idx_t i = 0; i < n; ++i) SA[i] = -1;
    for (idx_t i = 1; i < n; ++i)
        if (IS_LMS(t, i)) SA[--bkt[s[i]]] = i;
    induce(s, t, SA, n, K, bkt);

    idx_t n1 = 0;
    for (idx_t i = 0; i < n; ++i)
        if (IS_LMS(t, SA[i])) SA[n1++] = SA[i];

    /* name the sorted LMS substrings */
    for (idx_t i = n1; i < n; ++i) SA[i] = -1;
    idx_t name = 0, prev = -1;
    for (idx_t i = 0; i < n1; ++i) {
        const idx_t pos = SA[i];
        int diff = 0;
        for (idx_t d = 0; d < n; ++d) {
            if (prev == -1 || s[pos + d] != s[prev + d] || t[pos + d] != t[prev + d]) {
                diff = 1;
                break;
            }
            if (d > 0 && (IS_LMS(t, pos + d) || IS_LMS(t, prev + d))) break;
        }
        if (diff) { name++; prev = pos; }
        SA[n1 + pos / 2] = name - 1;
    }
    for (idx_t i = n - 1, j = n - 1; i >= n1; --i)
        if (SA[i] >= 0) SA[j--] = SA[i];

    /* stage 2: sort the reduced string */
    idx_t *s1 = SA + n - n1, *SA1 = SA;
    if (name < n1) {
        if (sais(s1, n1, name, SA1) != 0) { free(t); free(bkt); return -1; }
    } else {
        for (idx_t i = 0; i < n1; ++i) SA1[s1[i]] = i;
    }

    /* stage 3: induce the full order from the sorted LMS suffixes */
    bucket_bounds(s, n, K, bkt, 1);
    for (idx_t i = 1, j = 0; i < n; ++i)
        if (IS_LMS(t, i)) s1[j++] = i;
    for (idx_t i = 0; i < n1; ++i) SA1[i] = s1[SA1[i]];
    for (idx_t i = n1; i < n; ++i) SA[i] = -1;
    for (idx_t i = n1 - 1; i >= 0; --i) {
        const idx_t j = SA[i];
        SA[i] = -1;
        SA[--bkt[s[j]]] = j;
    }
    induce(s, t, SA, n, K, bkt);
    free(t);
    free(bkt);
    return 0;
}

int tpzh_suffix_array(const uint8_t *T, int64_t n, int64_t *SA) {
    if (n <= 0) return 0;
    idx_t *s = malloc(sizeof(idx_t) * (n + 1));
    idx_t *sa = malloc(sizeof(idx_t) * (n + 1));
    if (!s || !sa) { free(s); free(sa); return -1; }
    for (int64_t i = 0; i < n; ++i) s[i] = (idx_t)T[i] + 1;
    s[n] = 0;   /* sentinel, smaller than every byte */
    const int rc = sais(s, n + 1, 257, sa);
    if (rc == 0) memcpy(SA, sa + 1, sizeof(int64_t) * n);   /* sa[0] is the sentinel */
    free(s);
    free(sa);
    return rc;
}
