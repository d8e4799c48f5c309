/*
 * tpzh_main.c -- the `topaz` command line: `topaz index` and `topaz search`
 * with the options, defaults and error messages of src/main.c:15-340 (and
 * the defaults of src/options.h:6-23).  One extra long option, --batch N,
 * sets how many queries go to the device per batch.
 */
#define _GNU_SOURCE
#include "tpzh.h"

#include <errno.h>
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PROGRAM "topaz"

static void usage(void) {
    fprintf(stderr, "usage: %s <index|search> [-h] [-f FASTA] [-p STR]\n"
"\nGeneric:\n"
"\t-h, --help\n"
"\t-f FASTA, --file FASTA\n"
"\t-p STR, --prefix STR\n"
"\t-T INT, --threads INT (number of threads, default = %d)\n"
"\nOutput:\n"
"\t-H INT, --hits INT (default = %d)\n"
"\t-E FLOAT, --evalue FLOAT (default = %.1e)\n"
"\nAsymmetric SANS:\n"
"\t-S INT, --seeds INT (default = %d)\n"
"\t-A INT, --alignments INT (default = %d)\n"
"\t-l INT, --minlength INT (minimum length common substring, default = %d)\n"
"\t-s INT, --minscore INT (minimum raw score of common substring, default = %d)\n"
"\t-F, --fast (parameter defaults for 'fast' mode: seeds = %d, alignments = %d)"
"\nAlignment:\n"
"\t-o INT, --gapopen INT (default = %d)\n"
"\t-e INT, --gapext INT (default = %d)\n"
"\t-m STR, --matrix STR (substitution matrix, PAM*, BLOSUM*, default = %s)\n"
"\t-a FLOAT, --lambda FLOAT (E-value parameter, replace with lookup table like BLAST)\n"
"\t-k FLOAT, --kappa FLOAT (E-value parameter, replace with lookup table like BLAST)\n"
"\t-g FLOAT, --entropy FLOAT (E-value parameter, replace with lookup table like BLAST)\n"
"\t-B, --blasttab (output BLAST outfmt 6 tabular format at the expense of speed)\n"
"\t-M, --noseg (do not mask sequences with SEG during seeding)\n"
"\nB200:\n"
"\t--batch INT (queries per device batch, default = 2000)\n"
"\n", PROGRAM, 1, 100, 1e-3, 300000, 5000, 5, 1, 100000, 1500, 11, 1, "BLOSUM62");
}

/* str2sm (src/main.c:47-89): PAM30/70/250, BLOSUM45/50/62/80/90 by number */
static const char *matrix_name(const char *name) {
    static char buf[32];
    if (strncmp("PAM", name, 3) == 0) {
        const long v = strtol(name + 3, NULL, 10);
        if (v == 30 || v == 70 || v == 250) { snprintf(buf, sizeof buf, "PAM%ld", v); return buf; }
        return NULL;
    }
    if (strncmp("BLOSUM", name, 6) == 0) {
        const long v = strtol(name + 6, NULL, 10);
        if (v == 45 || v == 50 || v == 62 || v == 80 || v == 90) { snprintf(buf, sizeof buf, "BLOSUM%ld", v); return buf; }
    }
    return NULL;
}

#define INT_ARG(field, what)                                                                   \
    do {                                                                                       \
        field = strtol(optarg, &tmp, 10);                                                      \
        if (*tmp != '\0') {                                                                    \
            fprintf(stderr, "Error: invalid argument for --" what ", %s (%s)\n", strerror(errno), optarg); \
            exit(EXIT_FAILURE);                                                                \
        }                                                                                      \
    } while (0)

#define DBL_ARG(field, what)                                                                   \
    do {                                                                                       \
        field = strtod(optarg, &tmp);                                                          \
        if (tmp == optarg || *tmp != '\0') {                                                   \
            fprintf(stderr, "Error: invalid argument for --" what ", %s (%s)\n", strerror(errno), optarg); \
            exit(EXIT_FAILURE);                                                                \
        }                                                                                      \
    } while (0)

int tpzh_main(int argc, char **argv) {
    static struct option longopts[] = {
        {"help", no_argument, NULL, 'h'},           {"file", required_argument, NULL, 'f'},
        {"prefix", required_argument, NULL, 'p'},   {"threads", required_argument, NULL, 'T'},
        {"hits", required_argument, NULL, 'H'},     {"evalue", required_argument, NULL, 'E'},
        {"gapopen", required_argument, NULL, 'o'},  {"gapextend", required_argument, NULL, 'e'},
        {"matrix", required_argument, NULL, 'm'},   {"lambda", required_argument, NULL, 'a'},
        {"kappa", required_argument, NULL, 'k'},    {"entropy", required_argument, NULL, 'g'},
        {"minlength", required_argument, NULL, 'l'}, {"minscore", required_argument, NULL, 's'},
        {"blasttab", no_argument, NULL, 'B'},       {"alignments", required_argument, NULL, 'A'},
        {"seeds", required_argument, NULL, 'S'},    {"noseg", no_argument, NULL, 'M'},
        {"fast", no_argument, NULL, 'F'},           {"batch", required_argument, NULL, 1000},
        {0, 0, 0, 0}};
    if (argc < 2) { usage(); exit(EXIT_FAILURE); }
    int command;
    if (strcmp(argv[1], "index") == 0) command = 0;
    else if (strcmp(argv[1], "search") == 0) command = 1;
    else {
        if (strcmp(argv[1], "-h") != 0 && strcmp(argv[1], "--help") != 0) {
            fprintf(stderr, "Unrecognised command: '%s' (valid commands are 'index' and 'search')\n", argv[1]);
            exit(EXIT_FAILURE);
        }
        usage();
        exit(EXIT_SUCCESS);
    }
    tpzh_options o;
    tpzh_options_defaults(&o);
    char *fname = NULL, *prefix = NULL, *tmp = NULL;
    int c;
    while ((c = getopt_long(argc - 1, argv + 1, "hf:p:T:H:E:o:e:m:a:k:g:l:s:BA:S:MF", longopts, 0)) != -1) {
        switch (c) {
        case 'h': usage(); exit(EXIT_SUCCESS);
        case 'f': fname = optarg; break;
        case 'p': prefix = optarg; break;
        case 'H': INT_ARG(o.num_hits, "hits"); break;
        case 'o': INT_ARG(o.gap_open, "gapopen"); break;
        case 'e': INT_ARG(o.gap_extend, "gapextend"); break;
        case 'm':
            o.matrix = matrix_name(optarg);
            if (!o.matrix) {
                fprintf(stderr, "Error: invalid argument for --substitution, (\"%s\" is not the name of a substitution matrix)\n", optarg);
                exit(EXIT_FAILURE);
            }
            break;
        case 'E': DBL_ARG(o.evalue, "evalue"); break;
        case 'a': DBL_ARG(o.lambda, "lambda"); break;
        case 'k': DBL_ARG(o.k, "kappa"); break;
        case 'g': DBL_ARG(o.H, "entropy"); break;
        case 'l': INT_ARG(o.min_hit_length, "minlength"); break;
        case 's': INT_ARG(o.min_hit_score, "minscore"); break;
        case 'T': INT_ARG(o.num_threads, "threads"); break;
        case 'B': o.superfast = 0; break;
        case 'A': INT_ARG(o.number_of_alignments, "alignments"); break;
        case 'S': INT_ARG(o.number_of_seeds, "seeds"); break;
        case 'M': o.seg_enabled = 0; fprintf(stderr, "WARNING: SEG disabled\n"); break;
        case 'F':
            o.number_of_seeds = 100000;
            o.number_of_alignments = 1500;
            fprintf(stderr, "fast mode enabled\n");
            break;
        case 1000: INT_ARG(o.batch, "batch"); break;
        default: exit(EXIT_FAILURE);
        }
    }
    if (!fname) { fprintf(stderr, "ERROR: you must specify a FASTA file as input\n"); exit(EXIT_FAILURE); }
    if (!prefix) { fprintf(stderr, "ERROR: you must specify a database prefix\n"); exit(EXIT_FAILURE); }
    if (o.min_hit_length < 3) { fprintf(stderr, "ERROR: minimum seed length must be at least 3\n"); exit(EXIT_FAILURE); }
    if (o.number_of_alignments < 0) { fprintf(stderr, "ERROR: number of alignments must be positive\n"); exit(EXIT_FAILURE); }
    if (o.number_of_seeds < 0) { fprintf(stderr, "ERROR: number of seeds must be positive\n"); exit(EXIT_FAILURE); }
    if (command == 0) return tpzh_index(fname, prefix) == 0 ? EXIT_SUCCESS : EXIT_FAILURE;
    return tpzh_search(fname, prefix, &o) == 0 ? EXIT_SUCCESS : EXIT_FAILURE;
}
