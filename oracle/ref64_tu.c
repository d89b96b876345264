/*
 * ref64_tu.c -- builds the reference header with every float replaced by
 * double (TEST INFRASTRUCTURE ONLY).  System headers come first so that the
 * substitution only reaches CatmullClark.h itself.  The result is a loose
 * cross-check of the FP64 oracle: in this build crease sharpness is refined
 * in double as well.
 */
#include <stdint.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <assert.h>
#include <omp.h>
#define float double
#define CC_IMPLEMENTATION
#include "CatmullClark.h"
#undef float
void ccref64_set_threads(int n) { omp_set_num_threads(n); }
