/*
 * CPU ORACLE -- test infrastructure only.
 *
 * Link stubs for the logging hooks that the reference's matrix_cpu.c and
 * matrix_gpu.cu call (Error, source/xlog.c:424; Exit, source/xlog.c:891; Log and
 * Debug from the same file).  They only log in the reference; here Error only
 * counts and Log / Debug do nothing, so a batch run stays quiet.  Exit is
 * reached only when gsl_linalg_LU_decomp itself fails (not possible for the
 * square inputs this harness passes) or when a CUDA call of the cuSOLVER build
 * fails.
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

int
Log (const char *format, ...)
{
  (void) format;
  return 0;
}

int
Debug (const char *format, ...)
{
  (void) format;
  return 0;
}

long
ref_error_messages (void)
{
  return ref_error_count;
}
