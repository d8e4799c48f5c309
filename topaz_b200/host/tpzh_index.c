/*
 * tpzh_index.c -- `topaz index`: FASTA -> .pin/.psq/.phr (demultiplex_fasta,
 * src/demux.c:15-50), .SA/.ISA (serif_index, src/index.c:24-93) and .ind
 * (create_index, src/index.c:115-172).  Same file layouts byte for byte:
 *   .psq  internal-alphabet residues of every protein followed by '\n'
 *   .phr  every protein id followed by '\n'
 *   .pin  "psq_offset length phr_offset idlen\n" per protein
 *   .SA   little-endian int64 suffix array of the .psq bytes
 *   .ISA  zero-filled, same size as .SA
 *   .ind  packed {u64 header_start, u64 protein_start, i32 header_len,
 *         i32 protein_len} per protein
 */
#define _GNU_SOURCE
#include "tpzh.h"
#include "../../include/topaz_b200.h"

#include <errno.h>
#include <fcntl.h>
#include <inttypes.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

static char *fname(const char *prefix, const char *ext) {
    const size_t a = strlen(prefix), b = strlen(ext);
    char *s = malloc(a + b + 1);
    memcpy(s, prefix, a);
    memcpy(s + a, ext, b + 1);
    return s;
}

static FILE *open_w(const char *prefix, const char *ext) {
    char *n = fname(prefix, ext);
    FILE *f = fopen(n, "w");
    if (!f) fprintf(stderr, "Error: could not open %s, %s\n", n, strerror(errno));
    free(n);
    return f;
}

typedef struct {
    uint64_t header_start, protein_start;
    int32_t header_len, protein_len;
} ind_rec;

typedef struct {
    int fd;
    int err;     /* errno of a failed write */
} sa_file_t;

/* tpz_sa_build_sink's sink: rows [first_row, first_row + count) at their
 * offset in the .SA file */
static int sa_to_file(void *user, int64_t first_row, const int64_t *rows, int64_t count) {
    sa_file_t *f = (sa_file_t *)user;
    const char *p = (const char *)rows;
    size_t left = (size_t)count * 8;
    off_t at = (off_t)first_row * 8;
    while (left > 0) {
        const ssize_t w = pwrite(f->fd, p, left, at);
        if (w <= 0) { f->err = errno ? errno : EIO; return -1; }
        p += w; at += w; left -= (size_t)w;
    }
    return 0;
}

int tpzh_index(const char *fasta, const char *prefix) {
    /* ---- demultiplex */
    FILE *pin = open_w(prefix, ".pin"), *psq = open_w(prefix, ".psq"), *phr = open_w(prefix, ".phr");
    if (!pin || !psq || !phr) return -1;
    tpzh_fasta f;
    if (tpzh_fasta_open(&f, fasta) != 0) return -1;
    tpzh_record r;
    int rc;
    while ((rc = tpzh_fasta_next(&f, &r)) == 1) {
        fprintf(pin, "%ld %d %ld %d\n", ftell(psq), r.seq_len, ftell(phr), r.id_len);
        for (int i = 0; i < r.seq_len; ++i) r.seq[i] = tpzh_aa2internal(r.seq[i]);
        fprintf(phr, "%.*s\n", r.id_len, r.id);
        fprintf(psq, "%.*s\n", r.seq_len, r.seq);
        tpzh_record_free(&r);
    }
    if (rc < 0) return -1;
    fprintf(stderr, "Read %" PRIu64 " sequences from %s\n", f.count, fasta);
    tpzh_fasta_close(&f);
    fclose(phr);
    fclose(psq);
    fclose(pin);

    /* ---- suffix array of the .psq bytes */
    char *tn = fname(prefix, ".psq");
    FILE *tf = fopen(tn, "rb");
    if (!tf) { fprintf(stderr, "Error: problem opening %s\n", tn); return -1; }
    fseek(tf, 0, SEEK_END);
    const int64_t Tsize = ftell(tf);
    fseek(tf, 0, SEEK_SET);
    uint8_t *T = malloc(Tsize > 0 ? Tsize : 1);
    if (Tsize > 0 && fread(T, 1, Tsize, tf) != (size_t)Tsize) { fprintf(stderr, "Error: short read of %s\n", tn); return -1; }
    fclose(tf);
    fprintf(stderr, "mmapped T (%s), file size is %" PRId64 " bytes\n", tn, Tsize);
    free(tn);
    /* on the GPU, streamed into the .SA file piece by piece (the whole
     * array, 8 bytes per text byte, is never held in host memory) */
    char *san = fname(prefix, ".SA");
    const int safd = open(san, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (safd < 0) { fprintf(stderr, "Error: could not open %s, %s\n", san, strerror(errno)); return -1; }
    if (ftruncate(safd, Tsize * 8) != 0) { fprintf(stderr, "Error: could not size %s, %s\n", san, strerror(errno)); return -1; }
    sa_file_t out = {safd, 0};
    if (tpz_sa_build_sink(T, Tsize, sa_to_file, &out, 0, NULL) != 0) {
        fprintf(stderr, "Error: suffix array construction failed (%s)\n",
                out.err ? strerror(out.err) : tpz_last_error());
        return -1;
    }
    if (close(safd) != 0) { fprintf(stderr, "Error: could not write %s\n", san); return -1; }
    free(san);
    FILE *isa = open_w(prefix, ".ISA");
    if (!isa || ftruncate(fileno(isa), Tsize * 8) != 0) return -1;
    fclose(isa);
    free(T);

    /* ---- .ind from .pin */
    fprintf(stderr, "creating protein offset index...\n");
    char *hn = fname(prefix, ".phr");
    FILE *hf = fopen(hn, "rb");
    uint64_t Psize = 0;
    int c;
    while ((c = fgetc(hf)) != EOF) {
        if (c == '\0') break;
        if (c == '\n') Psize++;
    }
    fclose(hf);
    free(hn);
    char *pn = fname(prefix, ".pin");
    FILE *pf = fopen(pn, "r");
    ind_rec *ind = calloc(Psize ? Psize : 1, sizeof(ind_rec));
    char *line = NULL;
    size_t cap = 0;
    uint64_t ln = 0;
    while (getline(&line, &cap, pf) > 0) {
        uint64_t ps, hs;
        int pl, hl;
        const int nm = sscanf(line, "%" SCNu64 " %d %" SCNu64 " %d\n", &ps, &pl, &hs, &hl);
        if (nm != 4) {
            fprintf(stderr, "Error: line %" PRIu64 " of %s contained %d elements (expected 4)\n", ln + 1, pn, nm);
            return -1;
        }
        if (ln < Psize) {
            ind[ln].header_start = hs; ind[ln].protein_start = ps;
            ind[ln].header_len = hl; ind[ln].protein_len = pl;
        }
        ln++;
    }
    free(line);
    fclose(pf);
    if (ln != Psize) {
        fprintf(stderr, "Error: expected %" PRIu64 " index entries, but read %" PRIu64 " from %s\n", Psize, ln, pn);
        return -1;
    }
    free(pn);
    const uint64_t length = Psize ? ind[Psize - 1].protein_start + ind[Psize - 1].protein_len : 0;
    if ((uint64_t)Tsize != length + 1) {
        fprintf(stderr, "Error: index length is %" PRIu64 ", but T length is %" PRId64 " ...\n", length, Tsize);
        return -1;
    }
    FILE *inf = open_w(prefix, ".ind");
    if (!inf || fwrite(ind, sizeof(ind_rec), Psize, inf) != Psize) return -1;
    fclose(inf);
    free(ind);
    fprintf(stderr, "Done!\n");
    return 0;
}
