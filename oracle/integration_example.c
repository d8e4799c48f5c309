/* The code of INTEGRATION.md section 2, verbatim between the markers:
 * compiled by `make -C oracle relink` against the TOPAZ sources' headers
 * and include/topaz_b200.h, so that the snippet a maintainer copies into
 * src/engine.c is known to compile. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
/* BEGIN INTEGRATION SNIPPET */
#include "db.h"
#include "hit.h"
#include "options.h"
#include "topaz_b200.h"

/* once, after db_load (src/engine.c:46-58) */
static tpz_index *gpu_index_create(db_t *db) {
    tpz_index *ix = NULL;
    if (tpz_index_create((const uint8_t *)db->T, (int64_t)db->Tsize, (const int64_t *)db->SA,
                         db->index, (int64_t)db->Psize, &ix) != TPZ_OK) {
        fprintf(stderr, "Error: %s\n", tpz_last_error());
        exit(EXIT_FAILURE);
    }
    return ix;
}

/* per batch of n queries, residues after run_seg + seq_2internal
 * (src/engine.c:250-277) concatenated in qcat; hits[q] receives query q's
 * hitlist in traversal order (capacity opt->number_of_alignments, or
 * 1.5 * opt->num_hits for queries over 3000 residues), nhits[q] its size */
static void gpu_search_batch(tpz_index *ix, options_t *opt, const char *qcat,
                             const int64_t *qoff, const int32_t *qlen, int64_t n,
                             hit_t **hits, int64_t *nhits) {
    tpz_search_opts so;
    memset(&so, 0, sizeof so);
    so.num_hits = opt->num_hits;
    so.gap_open = opt->gap_open;
    so.gap_extend = opt->gap_extend;
    so.min_hit_length = opt->min_hit_length;
    so.seeds = opt->number_of_seeds;
    so.alignments = opt->number_of_alignments;
    so.mat625 = (const int8_t *)*opt->substitution;
    tpz_search_result *res = NULL;
    if (tpz_search_batch(ix, qcat, qoff, qlen, n, &so, &res) != TPZ_OK) {
        fprintf(stderr, "Error: %s\n", tpz_last_error());
        exit(EXIT_FAILURE);
    }
    for (int64_t q = 0; q < n; ++q) {
        nhits[q] = res->hit_off[q + 1] - res->hit_off[q];
        for (int64_t h = res->hit_off[q]; h < res->hit_off[q + 1]; ++h) {
            hit_t *t = &hits[q][h - res->hit_off[q]];
            memset(t, 0, sizeof *t);
            t->db_index = (uint64_t)res->protein[h];
            t->gapless_score = res->gapless_score[h];
            t->gapless_length = res->gapless_length[h];
            t->suffix_offset = res->suffix_offset[h];
            if (res->sw_status[h] == TPZ_SW_GAPLESS_LOW) {   /* ssw_wrapper.c:171-176 */
                t->is_aligned = 1;
                t->bitscore = 0;
                t->evalue = 1000;
            } else if (res->sw_status[h] == TPZ_SW_OK) {
                t->is_aligned = 1;
                t->rawscore = res->rawscore[h];
                t->qend = res->qend[h];
                t->send = res->send[h];
                tpz_karlin(qlen[q], opt->db_size, opt->db_proteins, opt->lambda, opt->k, opt->H,
                           t->rawscore, &t->bitscore, &t->evalue);
            } else {                                          /* dropped at 32767 */
                t->rawscore = 32767;
            }
        }
    }
    tpz_search_result_free(res);
}
/* END INTEGRATION SNIPPET */

/* keeps the static functions referenced */
void *integration_example_entry[] = {(void *)gpu_index_create, (void *)gpu_search_batch};
