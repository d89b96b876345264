/*
 * ref_extras.c -- two helpers linked beside the reference in oracle/_ref/.
 *
 * TEST INFRASTRUCTURE ONLY (part of the checker): lets the tests pick the
 * OpenMP thread count of the reference build (1 thread = the deterministic
 * order the FP32 oracle reproduces bit for bit; all cores = the timed CPU
 * baseline).
 */
#include <omp.h>

void ccref_set_threads(int n) { omp_set_num_threads(n); }
int ccref_max_threads(void) { return omp_get_max_threads(); }
