/*
 * oracle.h -- CPU restatement of the TOPAZ search hot path.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker.  The product never links it.
 *
 * Conventions shared with the product C-ABI (include/topaz_b200.h):
 *   - residues of queries and subjects for SW are substitution-matrix
 *     indices 0..24 in the order ARNDCQEGHILKMFPSTWYVBJZX*;
 *   - the DB text T and query strings for seeding are in TOPAZ's internal
 *     alphabet ('A'..'Y', '\n' delimiter);
 *   - matrices are 25x25 int8, row = subject letter, column = query letter.
 */
#ifndef TPZ_ORACLE_H
#define TPZ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Smith-Waterman with the striped-SSW result semantics ---- */
int orc_ssw_align(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                  const int8_t *mat25, int gap_open, int gap_extend,
                  int32_t *score, int32_t *ref_end, int32_t *read_end);
/* textbook Gotoh local alignment with the same tie rules (for comparison) */
int orc_gotoh_align(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                    const int8_t *mat25, int gap_open, int gap_extend,
                    int32_t *score, int32_t *ref_end, int32_t *read_end);
void orc_ssw_batch(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                   const int8_t *s, const int64_t *soff, const int32_t *slen,
                   const int8_t *mat25, int go, int ge, int nthreads,
                   int32_t *score, int32_t *ref_end, int32_t *read_end, int32_t *status);

/* ---- seeding ---- */
int64_t orc_lower_bound(const char *T, int64_t Tsize, const int64_t *SA,
                        const char *P, int64_t Psize);
void orc_hsp(const char *T, int64_t Tsize, const int64_t *SA, const char *Q, int32_t qlen,
             int32_t off, int64_t row, const int8_t *mat25, int32_t *score, int32_t *len);

/* ---- one whole query (seed -> walk -> hitlist -> SW -> rank) ---- */
typedef struct {
    int32_t num_hits;        /* -H */
    double evalue;           /* -E */
    int32_t gap_open, gap_extend;
    double lambda, k, H;
    int32_t min_hit_length;  /* -l */
    int32_t seeds;           /* -S */
    int32_t alignments;      /* -A */
} orc_opts_t;

typedef struct {
    int64_t db_index;
    int32_t gapless_score, gapless_length, suffix_offset, is_aligned;
    int32_t rawscore, qend, send, status;
    double bitscore, evalue;
} orc_hit_t;

/* Returns the number of hits (hitlist traversal order) or -1 on a read of the
 * SA past the zero-filled end page (where the reference faults). */
int orc_query_run(const char *T, int64_t Tsize, const int64_t *SA, const int64_t *pstart,
                  int64_t Psize, const char *qint, int32_t qlen, const int8_t *mat25,
                  const orc_opts_t *o, int64_t *pop_row, int32_t *pop_off, int32_t *pop_score,
                  int32_t *pop_len, int32_t *pop_counted, int64_t max_pops, int64_t *npops,
                  int64_t *ncounted, orc_hit_t *hits, int32_t max_hits);

/* Top-H selection of output_top_hits: indices into `hits` of the printed
 * lines, in print order.  Returns the count. */
int orc_rank_select(const orc_hit_t *hits, int32_t nhits, int32_t num_hits, double evalue,
                    int32_t *out_idx);

#ifdef __cplusplus
}
#endif
#endif
