/* relink_driver.c -- test infrastructure: drives the reference's own
 * get_ssw_profile / align_using_ssw_profile / stats_using_ssw_profile
 * (src/ssw_wrapper.c:105-245, compiled UNCHANGED) after they were relinked
 * against libtopaz_b200 in place of src/ssw.c, the way a maintainer would
 * relink the per-hit code (the shims of include/topaz_b200_ssw.h stand in
 * for SSW).  Built by `make -C oracle relink` into _ref/librelink.so.
 *
 * One call handles n (query, subject) pairs given in the internal alphabet
 * (what engine.c hands the wrapper after seq_2internal): per pair a seq_t of
 * each, a hit_t with the given gapless score, options_t with the given
 * matrix, gaps and Karlin-Altschul parameters -- the fields these functions
 * read (src/ssw_wrapper.c:105-245). */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "hit.h"
#include "options.h"
#include "seq.h"
#include "ssw_wrapper.h"

static seq_t *make_seq(const char *res, int32_t len) {
    seq_t *s = seq_alloc();
    seq_id(s, "x", 1);
    seq_seq(s, (char *)res, len, 0);
    return s;
}

/* out_i: n x 8 {rawscore, qend, send, qstart, sstart, length, mismatch,
 * gapopen}; out_d: n x 3 {bitscore, evalue, identity}.  rawscore 32767 is
 * the reference's dropped hit.  Returns 0. */
int relink_align(int64_t n, const char *qcat, const int64_t *qoff, const int32_t *qlen,
                 const char *scat, const int64_t *soff, const int32_t *slen,
                 const int8_t *mat625, int gap_open, int gap_extend, double lambda, double k,
                 double H, uint64_t db_size, uint64_t db_proteins, const int32_t *gapless,
                 int with_stats, int32_t *out_i, double *out_d) {
    int8_t mat[625];
    memcpy(mat, mat625, 625);
    options_t o;
    memset(&o, 0, sizeof o);
    o.substitution = (int8_t(*)[625])mat;
    o.gap_open = gap_open;
    o.gap_extend = gap_extend;
    o.lambda = lambda;
    o.k = k;
    o.H = H;
    o.db_size = db_size;
    o.db_proteins = db_proteins;
    o.evalue = 1e-3;
    for (int64_t i = 0; i < n; ++i) {
        seq_t *q = make_seq(qcat + qoff[i], qlen[i]);
        seq_t *s = make_seq(scat + soff[i], slen[i]);
        hit_t h;
        memset(&h, 0, sizeof h);
        h.gapless_score = gapless[i];
        h.qstart = h.sstart = h.length = h.mismatch = h.gapopen = -9;
        s_profile *p = get_ssw_profile(q, &o);
        align_using_ssw_profile(p, s, &h, &o);
        if (with_stats && h.gapless_score >= 40) stats_using_ssw_profile(p, s, &h, &o);
        init_destroy2(p);
        int32_t *oi = out_i + 8 * i;
        oi[0] = h.rawscore; oi[1] = h.qend; oi[2] = h.send; oi[3] = h.qstart;
        oi[4] = h.sstart; oi[5] = h.length; oi[6] = h.mismatch; oi[7] = h.gapopen;
        out_d[3 * i] = h.bitscore;
        out_d[3 * i + 1] = h.evalue;
        out_d[3 * i + 2] = h.identity;
        seq_free(q);
        seq_free(s);
    }
    return 0;
}
