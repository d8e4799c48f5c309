/*
 * topaz_b200_ssw.h -- the SSW calls TOPAZ makes per hit, under their own
 * names, as per-call shims over the B200 library (for parity tests and for
 * relinking the reference's per-hit code unchanged).
 *
 * Reference interface: src/ssw.h:87-210 (SSW 0.1.4 as vendored by TOPAZ);
 * callers get_ssw_profile / align_using_ssw_profile / stats_using_ssw_profile
 * (src/ssw_wrapper.c:105-245).  s_align keeps the SSW library's public field
 * layout and s_profile its public fields.  Supported as TOPAZ uses them:
 * score_size 2 (u8 pass, i16 rerun), n = 25, flag / filters / filterd
 * ignored (no begin positions or CIGAR: ref_begin1 = read_begin1 = -1,
 * cigar = NULL), no second-best alignment (score2 = 0, ref_end2 = -1).
 * ssw_align runs on the GPU (one launch for queries up to 1024 residues,
 * the batched kernels otherwise) and waits for its result; residues are
 * matrix indices 0..24 (host memory).
 */
#ifndef TOPAZ_B200_SSW_H
#define TOPAZ_B200_SSW_H

#include "topaz_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The query profile with the public fields of SSW's struct _profile
 * (src/ssw.h:31-40), so that callers reading them -- align_using_ssw_profile
 * reads readLen (src/ssw_wrapper.c:179-180) -- compile unchanged.  Here the
 * host SIMD profiles do not exist (NULL); the query and matrix live on the
 * device behind `device`, owned by the library. */
struct _profile {
    void *profile_byte;     /* NULL: no host u8 profile */
    void *profile_word;     /* NULL: no host i16 profile */
    int8_t *read;           /* as passed to ssw_init (init_destroy2 frees it) */
    const int8_t *mat;      /* the library's copy of the 25 x 25 matrix */
    int32_t readLen;
    int32_t n;              /* 25 */
    uint8_t bias;           /* -(smallest matrix entry), as ssw_init computes it */
    struct tpz_ssw_device *device;
};
typedef struct _profile s_profile;

typedef struct {
    uint16_t score1;
    uint16_t score2;
    int32_t ref_begin1;
    int32_t ref_end1;
    int32_t read_begin1;
    int32_t read_end1;
    int32_t ref_end2;
    uint32_t *cigar;
    int32_t cigarLen;
} s_align;

/* CIGAR words as BAM stores them (length << 4 | op; op 0..8 = "MIDNSHP=X"),
 * the helpers SSW's header provides inline (src/ssw.h:148-194).  No entry
 * point here produces a CIGAR; callers that print one still compile. */
#ifndef BAM_CIGAR_SHIFT
#define BAM_CIGAR_SHIFT 4
#endif
#ifndef MAPSTR
#define MAPSTR "MIDNSHP=X"
#endif
static inline uint32_t to_cigar_int(uint32_t length, char op_letter) {
    uint32_t op = 0;
    while (op < 9 && MAPSTR[op] != op_letter) ++op;
    return (length << BAM_CIGAR_SHIFT) | (op < 9 ? op : 0u);
}
static inline char cigar_int_to_op(uint32_t cigar_int) {
    const uint32_t op = cigar_int & 0xfu;
    return op < 9 ? MAPSTR[op] : 'M';
}
static inline uint32_t cigar_int_to_len(uint32_t cigar_int) { return cigar_int >> BAM_CIGAR_SHIFT; }

/* ssw_init (src/ssw.h:87): keeps `read` (init_destroy2 frees it, as
 * init_destroy2 does, src/ssw.c:828-833); NULL on bad arguments. */
TPZ_API s_profile *ssw_init(const int8_t *read, const int32_t readLen, const int8_t *mat,
                            const int32_t n, const int8_t score_size);
/* init_destroy / init_destroy2 (src/ssw.h:92-93) */
TPZ_API void init_destroy(s_profile *p);
TPZ_API void init_destroy2(s_profile *p);
/* ssw_align (src/ssw.h:128): NULL where the i16 pass reaches 32767 (the hit
 * is dropped, src/ssw_wrapper.c:222-226) or on an error. */
TPZ_API s_align *ssw_align(const s_profile *prof, const int8_t *ref, int32_t refLen,
                           const uint8_t weight_gapO, const uint8_t weight_gapE,
                           const uint8_t flag, const uint16_t filters, const int32_t filterd,
                           const int32_t maskLen);
/* align_destroy (src/ssw.h:141) */
TPZ_API void align_destroy(s_align *a);
/* ssw_align_stats (src/ssw.h:196-210, src/ssw.c:900-978): begin positions,
 * length, gap opens, mismatches and identity of the best alignment ending at
 * (read_end1, ref_end1) with score1; 1, or 0 after writing -1s on the
 * reference's guard. */
TPZ_API int ssw_align_stats(const s_profile *prof, const int8_t *ref, int32_t refLen,
                            const uint8_t weight_gapO, const uint8_t weight_gapE,
                            const int32_t maskLen, int32_t read_end1, int32_t ref_end1,
                            uint16_t score1, int32_t *read_begin1, int32_t *ref_begin1,
                            int32_t *length, int32_t *gapopen, int32_t *mismatch,
                            double *identity);

#ifdef __cplusplus
}
#endif
#endif
