/*
 * tpzh_fasta.c -- FASTA records and residue alphabets, with the record
 * splitting of TOPAZ's reader (src/fasta.c:62-120, src/seq.c:55-117).
 *
 * A record starts at a '>' that opens the file or follows '\n' and runs to
 * the byte before the next such '>'; the header is the record up to its
 * first '\n'; the residues are every later non-'\n' byte up to and including
 * the byte that ends the record span (for the last record, the file's last
 * byte), each passed through upper_aa.
 */
#define _GNU_SOURCE
#include "tpzh.h"

#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

char tpzh_upper_aa(char c) {
    if ((c >= 'A' && c <= 'Y') || c == '*' || c == '\n') return c;
    if (c >= 'a' && c <= 'y') return (char)(c - 32);
    return 'X';
}

/* internal alphabet: 'A'..'Y' stand for ACMLJIVTSKRQZEDBNHYFWXP*G */
char tpzh_aa2internal(char c) {
    static const char order[] = "ACMLJIVTSKRQZEDBNHYFWXP*G";
    if (c == '\n') return '\n';
    for (int i = 0; order[i]; ++i) {
        if (c == order[i]) return (char)('A' + i);
        if (c == order[i] + 32 && order[i] != '*') return (char)('a' + i);
    }
    return 'V';
}

int tpzh_header_id(const char *buf, int len, const char **id) {
    if (len <= 0) { *id = buf; return 0; }
    const int start = buf[0] == '>' ? 1 : 0;
    int i = start;
    while (i < len && buf[i] != ' ' && buf[i] != '\t') ++i;
    *id = buf + start;
    return i - start;
}

int tpzh_fasta_open(tpzh_fasta *f, const char *path) {
    memset(f, 0, sizeof *f);
    f->fd = open(path, O_RDONLY);
    struct stat sb;
    if (f->fd < 0 || fstat(f->fd, &sb) != 0) {
        fprintf(stderr, "Error: problem mapping %s\n", path);
        return -1;
    }
    f->size = (uint64_t)sb.st_size;
    if (f->size == 0) {
        fprintf(stderr, "Error: %s does not appear to be a FASTA file (first char not '>')\n", path);
        return -1;
    }
    f->data = mmap(NULL, f->size, PROT_READ, MAP_PRIVATE, f->fd, 0);
    if (f->data == MAP_FAILED) {
        f->data = NULL;
        fprintf(stderr, "Error: problem mapping %s\n", path);
        return -1;
    }
    madvise((void *)f->data, f->size, MADV_SEQUENTIAL);
    if (f->data[0] != '>') {
        fprintf(stderr, "Error: %s does not appear to be a FASTA file (first char not '>')\n", path);
        return -1;
    }
    return 0;
}

void tpzh_fasta_close(tpzh_fasta *f) {
    if (f->data) munmap((void *)f->data, f->size);
    if (f->fd > 0) close(f->fd);
    memset(f, 0, sizeof *f);
}

void tpzh_record_free(tpzh_record *r) {
    free(r->id);
    free(r->seq);
    memset(r, 0, sizeof *r);
}

int tpzh_fasta_next(tpzh_fasta *f, tpzh_record *r) {
    if (f->pos == f->size) return 0;
    uint64_t i;
    for (i = f->pos + 1; i < f->size + 1; ++i)
        if (i == f->size || (f->data[i - 1] == '\n' && f->data[i] == '>')) break;
    const char *rec = f->data + f->pos;
    const uint64_t len = i - f->pos - 1;
    const char *nl = memchr(rec, '\n', len);
    if (!nl) {
        fprintf(stderr, "Error: encountered a problem parsing FASTA file (%llu sequences were read without error)\n",
                (unsigned long long)f->count);
        return -1;
    }
    const uint64_t hdr = (uint64_t)(nl - rec);
    const char *id;
    const int idl = tpzh_header_id(rec, (int)hdr, &id);
    r->id = malloc(idl + 1);
    memcpy(r->id, id, idl);
    r->id[idl] = 0;
    r->id_len = idl;
    /* the residue span is len - hdr bytes starting after the newline */
    const uint64_t n = len - hdr;
    r->seq = malloc(n + 1);
    int k = 0;
    for (uint64_t j = 0; j < n; ++j) {
        const char c = nl[1 + j];
        if (c != '\n') r->seq[k++] = tpzh_upper_aa(c);
    }
    r->seq[k] = 0;
    r->seq_len = k;
    f->pos = i;
    f->count++;
    return 1;
}
