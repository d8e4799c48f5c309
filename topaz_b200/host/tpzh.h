/*
 * tpzh.h -- host side of the B200 TOPAZ search: CLI, FASTA, SEG, index
 * files, output.  Plain C; the device work goes through include/topaz_b200.h.
 */
#ifndef TPZH_H
#define TPZH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define TPZH_API __attribute__((visibility("default")))
#else
#define TPZH_API
#endif

/* ---------------------------------------------------------------- FASTA */
typedef struct {
    char *id;          /* header up to the first space/tab, '>' skipped */
    int id_len;
    char *seq;         /* residues, upper-cased by upper_aa */
    int seq_len;
} tpzh_record;

typedef struct {
    const char *data;
    uint64_t size, pos, count;
    int fd;
} tpzh_fasta;

/* returns 0, or -1 (message on stderr) when the file cannot be mapped or
 * does not start with '>' (src/fasta.c:17-51) */
TPZH_API int tpzh_fasta_open(tpzh_fasta *f, const char *path);
/* next record (src/fasta.c:62-120); 1 = got one, 0 = end, -1 = malformed */
TPZH_API int tpzh_fasta_next(tpzh_fasta *f, tpzh_record *r);
TPZH_API void tpzh_fasta_close(tpzh_fasta *f);
TPZH_API void tpzh_record_free(tpzh_record *r);

/* upper_aa (src/lexicographical.h:35-58) and aa2internal (:135-192) */
TPZH_API char tpzh_upper_aa(char c);
TPZH_API char tpzh_aa2internal(char c);
/* seq_id (src/seq.c:55-78): the id part of a header of `len` bytes */
TPZH_API int tpzh_header_id(const char *buf, int len, const char **id);

/* ------------------------------------------------------------------ SEG */
/* hard-masks low-complexity regions of upper-cased residues with 'X'
 * (run_seg, src/seg_wrapper.c:15-49); returns the number of segments */
TPZH_API int tpzh_seg_mask(char *seq, int len);
/* the tables the device SEG computes with (ent_full 13, logxr 13 x 13,
 * lnfac n entries), from the same functions as tpzh_seg_mask */
TPZH_API void tpzh_seg_tables(double *ent_full, double *logxr, double *lnfac_out, int n);

/* ---------------------------------------------------------------- index */
/* `topaz index -f FASTA -p PREFIX` (serif_index, src/index.c:24-93) */
TPZH_API int tpzh_index(const char *fasta, const char *prefix);

/* -------------------------------------------------- blasttab statistics */
typedef struct {
    int32_t qstart, sstart, length, mismatch, gapopen;
    double identity;
} tpzh_stats;

/* ssw_align_stats (src/ssw.c:900-978) for one printed hit: query/subject as
 * matrix indices, the forward result (score, read_end, ref_end). */
TPZH_API int tpzh_align_stats(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                              const int8_t *mat625, int gap_open, int gap_extend,
                              int32_t read_end1, int32_t ref_end1, int32_t score1,
                              tpzh_stats *out);

/* ---------------------------------------------------------------- search */
typedef struct {
    int num_threads, num_hits, gap_open, gap_extend, min_hit_length, min_hit_score;
    int number_of_alignments, number_of_seeds, seg_enabled, superfast;
    double evalue, lambda, k, H;
    const char *matrix;
    int64_t batch;     /* queries per device batch */
} tpzh_options;

TPZH_API void tpzh_options_defaults(tpzh_options *o);
TPZH_API int tpzh_search(const char *fasta, const char *prefix, const tpzh_options *o);

/* CLI entry (src/main.c:111-340) */
TPZH_API int tpzh_main(int argc, char **argv);

#ifdef __cplusplus
}
#endif
#endif
