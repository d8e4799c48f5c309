/*
 * topaz_b200.h -- C ABI of the B200-native TOPAZ search hot path.
 *
 * Plain C types only (pointers, sizes, ints).  All functions return 0 on
 * success or a negative TPZ_E* code; tpz_last_error() gives a message.
 * "Device" entry points take CUDA device pointers and a cudaStream_t passed
 * as void* (NULL = legacy default stream) and only enqueue work; "host"
 * entry points take host buffers and return when the results are in them.
 *
 * Residues handed to Smith-Waterman are substitution-matrix indices 0..24 in
 * the order ARNDCQEGHILKMFPSTWYVBJZX* (what align_using_ssw_profile feeds
 * ssw_align after aa_table2, src/ssw_wrapper.c:113-120, :193-201).
 */
#ifndef TOPAZ_B200_H
#define TOPAZ_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define TPZ_API __attribute__((visibility("default")))
#else
#define TPZ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TPZ_OK = 0,
    TPZ_E_ARG = -1,        /* invalid argument (bad size, NULL, gap_open <= gap_extend) */
    TPZ_E_CUDA = -2,       /* a CUDA runtime call failed */
    TPZ_E_NOMEM = -3,      /* device memory could not be allocated */
    TPZ_E_RANGE = -4,      /* input beyond a stated maximum */
    TPZ_E_NODEV = -5,      /* no CUDA device */
    TPZ_E_DEVICE = -6      /* a kernel reported an error status (bounded wait expired, bad index) */
};

/* Per-pair status written by the SW entry points. */
enum {
    TPZ_SW_OK = 0,         /* score/ref_end/read_end valid */
    TPZ_SW_DROPPED = 1,    /* 16-bit score reached 32767: ssw_align returns NULL and the
                              hit is dropped (src/ssw.c:866-870, src/ssw_wrapper.c:222-226) */
    TPZ_SW_INVALID = 2,    /* pair outside the stated limits; not aligned */
    TPZ_SW_GAPLESS_LOW = 3 /* search hit with gapless score < 40: no SW, bitscore 0,
                              E-value 1000 (src/ssw_wrapper.c:171-176) */
};

/* Per-query status bits of tpz_search_batch. */
enum {
    TPZ_Q_SA_END = 1,      /* the walk reached a suffix-array row past the zero-filled
                              last page of the .SA mapping, where the reference reads
                              unmapped memory; the query stopped there */
    TPZ_Q_TOO_LONG = 2     /* query longer than TPZ_SEARCH_MAX_QLEN: not searched */
};

TPZ_API const char *tpz_last_error(void);

/* Creates the CUDA context of the current device and sets up the device
 * memory pool (no reference counterpart).  Optional: every entry point does
 * this on first use; a program can call it early on a thread of its own so
 * the start-up cost overlaps reading its input (`topaz search` does). */
TPZ_API int tpz_device_init(void);
TPZ_API const char *tpz_version(void);

/* Substitution matrix by name: BLOSUM45/50/62/80/90, PAM30/70/250
 * (str2sm, src/main.c:47-89).  Copies 625 int8 (row = subject letter) into
 * out.  Returns TPZ_E_ARG for an unknown name. */
TPZ_API int tpz_matrix(const char *name, int8_t *out625);

/* ------------------------------------------------------------------------
 * Batched Smith-Waterman: scores and end coordinates of n independent
 * (query, subject) pairs with exactly the results of
 *   ssw_init(query, qlen, mat, 25, 2) + ssw_align(prof, subject, slen,
 *   gap_open, gap_extend, 0, 0, 0, 15)            (src/ssw.c:799-897)
 * i.e. the u8 pass, its i16 rerun on saturation, and the drop at 32767.
 * Replaces the per-hit calls in perform_alignment_with_profile
 * (src/query.c:304-340) / align_using_ssw_profile (src/ssw_wrapper.c:157-245).
 *
 * Pair i: query = q[qoff[i] .. qoff[i]+qlen[i]), subject = s[soff[i] ..
 * soff[i]+slen[i]).  Limits: 1 <= qlen <= TPZ_SW_MAX_QLEN, 0 <= slen <
 * TPZ_SW_MAX_SLEN, gap_open > gap_extend >= 0, gap_open <= 255.
 * Outputs per pair: score, ref_end (0-based subject end, -1 when score is 0),
 * read_end (0-based query end), status (TPZ_SW_*).
 * ------------------------------------------------------------------------ */
#define TPZ_SW_MAX_QLEN 8192
#define TPZ_SW_MAX_SLEN (1 << 24)

TPZ_API int tpz_sw_batch_device(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                        const int8_t *s, const int64_t *soff, const int32_t *slen,
                        const int8_t *mat625_host, int gap_open, int gap_extend,
                        int32_t *score, int32_t *ref_end, int32_t *read_end, int32_t *status,
                        void *stream);

TPZ_API int tpz_sw_batch_host(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                      const int8_t *s, const int64_t *soff, const int32_t *slen,
                      const int8_t *mat625, int gap_open, int gap_extend,
                      int32_t *score, int32_t *ref_end, int32_t *read_end, int32_t *status);

/* One pair, one kernel launch: the per-pair form of ssw_init + ssw_align
 * (src/ssw_wrapper.c:157-245 calls them once per hit), with the same results
 * as tpz_sw_batch_device.  q, s and out4 are device pointers (q and s in
 * matrix-index residues, out4 = {score, ref_end, read_end, status}); the
 * launch goes on `stream` and the call does not wait for it.  Limits:
 * 1 <= qlen <= 1024, and qlen * (largest matrix entry) < 32512. */
TPZ_API int tpz_sw_align_one(const int8_t *q, int32_t qlen, const int8_t *s, int32_t slen,
                             const int8_t *mat625_host, int gap_open, int gap_extend,
                             int32_t *out4, void *stream);

/* Allocation-free variant of tpz_sw_batch_device, with no counterpart in the
 * TOPAZ reference.  For callers that must not have device memory allocated
 * on their behalf -- e.g. a server whose HBM is planned around a resident
 * index and fixed in-flight batches, where an allocation could fail midway
 * through a request, or a loop that cannot afford the device-wide
 * synchronization of cudaMalloc/cudaFree.  Same arguments and results as
 * tpz_sw_batch_device; at most TPZ_SW_NOALLOC_MAX_PAIRS pairs per call
 * (TPZ_E_RANGE beyond), queries of at most TPZ_SW_NOALLOC_MAX_QLEN
 * residues (longer ones get status TPZ_SW_INVALID) and matrices whose
 * largest entry is at most TPZ_SW_NOALLOC_MAX_ENTRY (TPZ_E_ARG beyond: such
 * scores can pass the 16-bit range, and the allocating call's 32-bit rerun
 * needs scratch of its own).  Scratch is one static device array per device
 * (about 0.6 MB, held until the process exits) shared by all calls: calls
 * whose work overlaps on the GPU (other streams or threads) race on it, so
 * order them on one stream.  All work goes to `stream`; nothing is
 * allocated or freed.  The first call on a device does a one-time set-up
 * (device address of the scratch array, kernel attributes) and should come
 * before any stream capture that includes a call. */
#define TPZ_SW_NOALLOC_MAX_PAIRS 65536
#define TPZ_SW_NOALLOC_MAX_QLEN 1024
#define TPZ_SW_NOALLOC_MAX_ENTRY 31
TPZ_API int tpz_sw_batch_device_noalloc(int64_t n, const int8_t *q, const int64_t *qoff,
                                        const int32_t *qlen, const int8_t *s, const int64_t *soff,
                                        const int32_t *slen, const int8_t *mat625_host,
                                        int gap_open, int gap_extend, int32_t *score,
                                        int32_t *ref_end, int32_t *read_end, int32_t *status,
                                        void *stream);

/* The --blasttab columns of n aligned pairs on the device: what
 * ssw_align_stats (src/ssw.c:900-978) computes for a hit whose forward pass
 * gave (score, read_end, ref_end) -- query and subject starts from a reverse
 * pass, then length, gap opens, mismatches and identity from the banded
 * alignment's path (src/ssw.c:538-784).  Pairs as tpz_sw_batch_device
 * (device buffers, matrix-index residues); read_end/ref_end/score per pair;
 * outputs per pair; -1 columns (identity -1.0) where the reference gives
 * them (no end cell, no start found, the band table's size guard).  Work
 * goes on `stream`; the call waits for it (it sizes scratch from the
 * device's results). */
TPZ_API int tpz_sw_stats_device(int64_t n, const int8_t *q, const int64_t *qoff,
                                const int32_t *qlen, const int8_t *s, const int64_t *soff,
                                const int32_t *slen, const int8_t *mat625_host, int gap_open,
                                int gap_extend, const int32_t *read_end, const int32_t *ref_end,
                                const int32_t *score, int32_t *qstart, int32_t *sstart,
                                int32_t *length, int32_t *gapopen, int32_t *mismatch,
                                double *identity, void *stream);

/* Kernel launches enqueued by the last tpz_sw_batch_* call on this thread
 * (for launch accounting). */
TPZ_API int64_t tpz_sw_last_launches(void);

/* ------------------------------------------------------------------------
 * Resident index: the .psq text, .SA and .ind of one database copied into
 * device memory once (db_load, src/db.c:34-126) plus derived tables.
 * T: Tsize bytes (internal alphabet, '\n' after every protein); SA: Tsize
 * int64; ind: Psize packed 24-byte records {u64 header_start, u64
 * protein_start, i32 header_len, i32 protein_len} (src/db.h:10-17).
 * Returns TPZ_E_ARG when the three do not describe one database.
 * ------------------------------------------------------------------------ */
typedef struct tpz_index tpz_index;

TPZ_API int tpz_index_create(const uint8_t *T, int64_t Tsize, const int64_t *SA, const void *ind,
                             int64_t Psize, tpz_index **out);
TPZ_API void tpz_index_destroy(tpz_index *ix);
TPZ_API int64_t tpz_index_device_bytes(const tpz_index *ix);

/* sa_search (src/search.c:237-362, declared src/search.h:14) for n whole
 * patterns pcat[poff[i] .. +plen[i]) (internal alphabet letters, plen >= 1):
 * idx[i] = the lower bound = number of suffixes smaller than the pattern. */
TPZ_API int tpz_sa_search_batch(const tpz_index *ix, const char *pcat, const int64_t *poff,
                                const int32_t *plen, int64_t n, int64_t *idx);

/* sa_hsp (src/search.c:99-190, declared src/search.h:13) for n (query,
 * offset, SA row) triples: score/length of the two-sided gapless extension;
 * length -1 when the first symbols differ (score then 0), -2 for a row
 * outside the readable SA. */
TPZ_API int tpz_sa_hsp_batch(const tpz_index *ix, const char *qcat, const int64_t *qoff,
                             const int32_t *qlen, int64_t nq, const int32_t *query_of,
                             const int32_t *qoffset, const int64_t *row, int64_t n,
                             const int8_t *mat625, int32_t *score, int32_t *length);

/* Per-call forms of the two seams, with the argument lists of
 * src/search.h:13-14: the resident index stands in for db_t (its T, SA and
 * Tsize), the query's residues and length for seq_t, the substitution
 * matrix for options_t (the one option sa_hsp reads).  Each call is one
 * small launch that waits for its result -- for parity tests and for
 * per-call sites; the batch forms above are the fast path.
 *
 * tpz_sa_search (sa_search, src/search.c:237-362): pattern = q[offset ..
 * offset + length), or to the end of q when length <= 0.  idx = the first row
 * whose suffix starts with the pattern if one does, else the lower bound;
 * num_matches = the number of rows starting with it; last_position = the
 * common prefix length with the last row the reference's first binary
 * search compares (the pattern length when a row starts with it).  Returns
 * 0, or -1 (with *idx = -1) for an empty pattern or index, as sa_search
 * does; TPZ_E_ARG for bytes outside 'A'..'Y'. */
TPZ_API int tpz_sa_search(const tpz_index *db, const char *q, int32_t qlen, int64_t offset,
                          int64_t length, int64_t *idx, int64_t *num_matches,
                          int64_t *last_position);
/* tpz_sa_hsp (sa_hsp, src/search.c:99-190): gapless extension of query
 * offset qoffset against SA row `position`; gapless_length -1 when the first
 * symbols differ, -2 for a row outside the readable SA (where sa_hsp reads
 * past its mapping).  Returns 0 as sa_hsp does, or a TPZ_E* code for bad
 * arguments (0 <= qoffset < qlen). */
TPZ_API int tpz_sa_hsp(const tpz_index *db, const char *q, int32_t qlen, int32_t qoffset,
                       int64_t position, const int8_t *mat625, int32_t *gapless_score,
                       int32_t *gapless_length);

/* ------------------------------------------------------------------------
 * Whole queries: seed lookup, best-first SA walk into the capped hitlist
 * and Smith-Waterman of every hit with gapless score >= 40 -- the work of
 * query_find_suffixes, query_fetch_alignment_batch and
 * query_perform_alignments (src/query.c:94-248) for a batch of queries
 * (internal alphabet, as after run_seg + seq_2internal, src/engine.c:250-277).
 * Hits come back per query in hitlist traversal order (gapless score
 * descending, newest first; src/rbtree.c:653-669) with E-values and ranking
 * left to the caller (tpz_karlin, output_top_hits), or, in report mode,
 * ranked and cut on the device.
 * ------------------------------------------------------------------------ */
#define TPZ_SEARCH_MAX_QLEN 8192

typedef struct {
    int32_t num_hits;         /* -H (hitlist capacity 1.5*H for queries > 3000) */
    int32_t gap_open;         /* -o */
    int32_t gap_extend;       /* -e */
    int32_t min_hit_length;   /* -l */
    int32_t seeds;            /* -S: counted pops per query */
    int32_t alignments;       /* -A: hitlist capacity */
    const int8_t *mat625;     /* substitution matrix (host) */
    int64_t trace_pops;       /* record up to this many pops per query (0: none) */
    /* Report mode (report_hits > 0): the ranking of output_top_hits
     * (src/engine.c:193-248) on the device.  Each query's aligned hits (SW
     * score, or gapless score < 40 with bitscore 0 and E-value 1000) are
     * stably sorted by bitscore descending, the first report_hits are kept and
     * those with E-value > max_evalue dropped; only these come back, in that
     * order, with bitscore and E-value.  Scores use tpz_karlin with the
     * parameters below (src/ssw_wrapper.c:179-183).  0: every hit comes back
     * in traversal order without E-values. */
    int32_t report_hits;      /* -H */
    double max_evalue;        /* -E */
    double lambda, k, H;      /* Karlin-Altschul parameters (0.267, 0.041, 0.140) */
    uint64_t db_size, db_proteins;
    /* report mode only: 1 = also the --blasttab columns of every reported
     * hit on the device (ssw_align_stats, src/ssw.c:900-978) */
    int32_t blasttab_stats;
    /* 0: queries come in the internal alphabet (after run_seg +
     * seq_2internal); 1: they come as upper-case residues and are SEG-masked
     * and mapped on the device (tpz_prepare_queries_device); 2: the same
     * without SEG (-M) */
    int32_t ingest;
} tpz_search_opts;

typedef struct {
    int64_t nq, nhits_total;
    const int64_t *hit_off;                  /* nq + 1 */
    const int64_t *npops, *ncounted;         /* nq */
    const int32_t *status;                   /* nq, TPZ_Q_* bits */
    const int32_t *protein, *gapless_score, *gapless_length, *suffix_offset;
    const int32_t *rawscore, *qend, *send, *sw_status;   /* per hit, TPZ_SW_* */
    const int64_t *trace_n;                  /* nq (when trace_pops > 0) */
    const int64_t *trace_row;                /* nq * trace_pops */
    const int32_t *trace_off, *trace_score, *trace_len, *trace_counted;
    double stage_ms[4];      /* device time: seed lookup, walk + hitlist, SW of hits
                                (+ ranking in report mode); [3] = host wall time of
                                the whole call incl. copies */
    const double *bitscore, *evalue;         /* per hit, report mode only (else NULL) */
    int64_t sw_pairs, sw_cells;              /* SW of hits: pairs, sum of qlen * slen */
    double seed_ms, chain_ms;                /* stage_ms[0] split: seed lookup, cursor chains */
    int64_t positions;                       /* query positions searched */
    /* per reported hit when opts.blasttab_stats (else NULL): 0-based query
     * and subject starts, alignment length, gap opens, mismatches, identity;
     * -1 columns for hits without a Smith-Waterman alignment */
    const int32_t *qstart, *sstart, *length, *gapopen, *mismatch;
    const double *identity;
    /* gapless extensions (sa_hsp) of the cursor chains: precomputed for
     * every queued cursor, and refilled by the walk */
    int64_t chain_elems, refill_elems;
} tpz_search_result;

TPZ_API int tpz_search_batch(const tpz_index *ix, const char *qcat, const int64_t *qoff,
                             const int32_t *qlen, int64_t nq, const tpz_search_opts *opts,
                             tpz_search_result **out);
TPZ_API void tpz_search_result_free(tpz_search_result *r);

/* Upper estimate of the device memory one query of length qlen takes inside
 * tpz_search_batch with options o (no reference counterpart): for callers
 * that admit queries against a memory budget (a serving loop).  -1 on bad
 * arguments. */
TPZ_API int64_t tpz_search_query_device_bytes(int32_t qlen, const tpz_search_opts *o);

/* Query ingest of a batch, in place (run_seg + seq_2internal,
 * src/engine.c:250-277): query i = cat[off[i] .. off[i]+len[i]) holds
 * upper-case residues (as the FASTA reader gives them); with seg != 0 SEG
 * hard-masks it (seg_wrapper.c:15-49), then every residue becomes its
 * internal-alphabet letter, the form tpz_search_batch takes.  Runs on
 * nthreads host threads. */
TPZ_API int tpz_prepare_queries(char *cat, const int64_t *off, const int32_t *len, int64_t n,
                                int seg, int nthreads);

/* The same ingest on the device, in place: query i = cat[off[i] ..
 * off[i]+len[i]) in device memory (upper-case residues in, internal
 * alphabet out; queries disjoint, total_bytes = the extent of cat they
 * use).  SEG's doubles are computed from the host's tables with separately
 * rounded operations, so the masks equal tpz_prepare_queries' bit for bit.
 * Work goes on `stream`; the call waits for it. */
TPZ_API int tpz_prepare_queries_device(char *cat, const int64_t *off, const int32_t *len,
                                       int64_t n, int64_t total_bytes, int seg, void *stream);

/* Suffix array of the .psq bytes T[0, n) on the device, for `topaz index`
 * (divsufsort64 in serif_index, src/index.c:24-93, builds it on the host):
 * SA[0, n) (host) receives the suffixes in byte-lexicographic order, a
 * shorter suffix before a longer one with the same prefix -- the bytes of the
 * reference's .SA file.  rounds (may be NULL) receives the number of sorting
 * rounds.  64-bit positions; the text, its inverse array (8 bytes per
 * position) and the sort buffers must fit in device memory (about 10 G
 * residues on one B200); TPZ_E_RANGE for texts where more suffixes share
 * their first few symbols than one device sort holds. */
TPZ_API int tpz_sa_build(const uint8_t *T, int64_t n, int64_t *SA, int32_t *rounds);

/* The same with the rows handed to a sink instead of one host array, so the
 * caller never holds the whole array (8 bytes per text byte) in memory:
 * sink(user, first_row, rows, count) receives SA[first_row .. first_row +
 * count); rows come mostly in increasing order, and rows inside long repeats
 * come again at the end with their final values (a file sink writes each
 * piece at its offset).  A nonzero return from the sink stops the build
 * (TPZ_E_ARG).  max_partition > 0 caps the suffixes sorted at once (0: as
 * the free device memory allows). */
typedef int (*tpz_sa_sink)(void *user, int64_t first_row, const int64_t *rows, int64_t count);
TPZ_API int tpz_sa_build_sink(const uint8_t *T, int64_t n, tpz_sa_sink sink, void *user,
                              int64_t max_partition, int32_t *rounds);

/* bitscore and E-value of a raw score exactly as align_using_ssw_profile
 * computes them with the C library's log/exp (src/ssw_wrapper.c:179-183,
 * :239-242); db_size = Tsize - Psize and db_proteins = Psize unless given
 * (src/engine.c:52-58). */
TPZ_API void tpz_karlin(int32_t qlen, uint64_t db_size, uint64_t db_proteins, double lambda,
                        double k, double H, int32_t raw, double *bitscore, double *evalue);

/* Roofline probe (no reference counterpart): `blocks` x 256 threads, each
 * running 8 independent chains of `iters` __viaddmax_s16x2 ops; writes one
 * word per thread to out (device, blocks*256 uint32) and the number of DPX
 * ops enqueued to *ops (host).  Timed by the caller on `stream`. */
TPZ_API int tpz_dpx_probe(int64_t blocks, int iters, uint32_t *out, void *stream, int64_t *ops);

#ifdef __cplusplus
}
#endif
#endif
