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
    TPZ_SW_INVALID = 2     /* pair outside the stated limits; not aligned */
};

TPZ_API const char *tpz_last_error(void);
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
 * soff[i]+slen[i]).  Limits: 1 <= qlen <= TPZ_SW_MAX_QLEN, 0 <= slen <=
 * TPZ_SW_MAX_SLEN, gap_open > gap_extend >= 0, gap_open <= 255.
 * Outputs per pair: score, ref_end (0-based subject end, -1 when score is 0),
 * read_end (0-based query end), status (TPZ_SW_*).
 * ------------------------------------------------------------------------ */
#define TPZ_SW_MAX_QLEN 1024
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

/* Kernel launches enqueued by the last tpz_sw_batch_* call on this thread
 * (for launch accounting). */
TPZ_API int64_t tpz_sw_last_launches(void);

/* Roofline probe (no reference counterpart): `blocks` x 256 threads, each
 * running 8 independent chains of `iters` __viaddmax_s16x2 ops; writes one
 * word per thread to out (device, blocks*256 uint32) and the number of DPX
 * ops enqueued to *ops (host).  Timed by the caller on `stream`. */
TPZ_API int tpz_dpx_probe(int64_t blocks, int iters, uint32_t *out, void *stream, int64_t *ops);

#ifdef __cplusplus
}
#endif
#endif
