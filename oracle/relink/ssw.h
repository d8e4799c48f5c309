/* Stands in for the TOPAZ source tree's ssw.h when the reference's
 * ssw_wrapper.c is compiled unchanged against this library (make -C oracle
 * relink): the SSW calls resolve to the B200 library's per-call shims. */
#include "topaz_b200_ssw.h"
