/* The reference's ExportToObj (examples/subd_cpu.c:22-115), compiled from its
 * own source for the tests (test infrastructure only): the example program
 * is included with its main renamed, and the static exporter is exposed as
 * ccref_export_obj.  Built twice by oracle/Makefile: as is (16-byte records)
 * and with -DCC_DISABLE_UV (12-byte records). */
#define main ccref_subd_cpu_main
#include "subd_cpu.c"
#undef main

void ccref_export_obj(const cc_Subd *subd, int32_t depth, const char *filename)
{
    ExportToObj(subd, depth, filename);
}
