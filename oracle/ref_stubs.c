/*
 * CPU ORACLE -- test infrastructure only.
 *
 * Link stubs for the two logging hooks that the reference's matrix_cpu.c
 * calls (Error, source/xlog.c:424; Exit, source/xlog.c:891).  Error only logs
 * in the reference; here it only counts, so a batch run stays quiet.  Exit is
 * reached only when gsl_linalg_LU_decomp itself fails, which cannot happen for
 * the square inputs this harness passes.
 */
#include <stdarg.h>
#include <stdlib.h>

static volatile long ref_error_count = 0;

int
Error (const char *format, ...)
{
  (void) format;
  __atomic_add_fetch (&ref_error_count, 1, __ATOMIC_RELAXED);
  return 0;
}

int
Exit (int error_code)
{
  exit (error_code);
  return 0;
}

long
ref_error_messages (void)
{
  return ref_error_count;
}
