/*
 * Build shim for the drop-in check (TEST INFRASTRUCTURE ONLY).  Placed first
 * on the include path when oracle/Makefile compiles the reference's own
 * examples/subd_cpu.c, it stands for that program's one added line: the
 * reference's CatmullClark.h (the next one on the path), then
 * include/ccs_cuda_compat.h, which from there on runs the program's subd
 * calls on the GPU through libccs_cuda.so.  The program's source is compiled
 * where it lies, unchanged.
 */
#include_next "CatmullClark.h"
#include "ccs_cuda_compat.h"
