/* topaz -- command line entry point (see tpzh_main.c) */
#include "tpzh.h"

int main(int argc, char **argv) { return tpzh_main(argc, argv); }
