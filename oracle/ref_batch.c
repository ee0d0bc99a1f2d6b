/*
 * CPU ORACLE -- test infrastructure only.
 *
 * Batch driver around a serial solve_matrix / invert_matrix pair, compiled
 * twice by oracle/Makefile:
 *   - against the reference's own source/matrix_cpu.c + vendored GSL 2.6
 *     (oracle/_ref/libref_matrix.so, symbols prefixed ref_), and
 *   - against the restatement in gsl_lu_oracle.c
 *     (oracle/_build/liboracle.so, symbols prefixed port_).
 * Each pthread walks a static contiguous share of the systems and calls the
 * serial routine once per system, the way one MPI rank of the reference calls
 * it once per plasma cell (source/macro_accelerate.c:1054-1061,
 * source/matrix_ion.c:276).  A is copied into a per-thread scratch before each
 * call because the reference factorises it in place (matrix_cpu.c:133).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef DRV_PREFIX
#error "DRV_PREFIX must name the exported symbol prefix"
#endif
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define EXPORT(name) CAT(DRV_PREFIX, name)

#ifdef DRV_USE_REFERENCE
/* reference prototypes, source/templates.h:358-360 */
int solve_matrix (double *a_matrix, double *b_matrix, int size, double *x_matrix, int nplasma);
int invert_matrix (double *matrix, double *inverted_matrix, int num_rows);
const char *get_matrix_error_string (int error_code);
void gsl_set_error_handler_off (void);
#define SOLVE(a, b, n, x, cell) solve_matrix ((a), (double *) (b), (n), (x), (cell))
#define INVERT(a, inv, n) invert_matrix ((a), (inv), (n))
#define ERRSTR(c) get_matrix_error_string (c)
#define PREPARE() gsl_set_error_handler_off ()
#else
int oracle_solve_matrix (double *a, const double *b, int n, double *x);
int oracle_invert_matrix (double *a, double *inv, int n);
const char *oracle_matrix_error_string (int code);
#define SOLVE(a, b, n, x, cell) oracle_solve_matrix ((a), (b), (n), (x))
#define INVERT(a, inv, n) oracle_invert_matrix ((a), (inv), (n))
#define ERRSTR(c) oracle_matrix_error_string (c)
#define PREPARE() ((void) 0)
#endif

typedef struct
{
  int kind;                     /* 0 solve, 1 invert */
  int lo, hi;
  const int *n;
  const int64_t *offA;
  const double *A;
  const int64_t *offv;
  const double *b;
  double *out;
  int *status;
} job_t;

static void *
run_job (void *arg)
{
  job_t *jb = (job_t *) arg;
  int nmax = 0;
  for (int s = jb->lo; s < jb->hi; s++)
    if (jb->n[s] > nmax)
      nmax = jb->n[s];
  double *scratch = (double *) malloc ((size_t) (nmax > 0 ? nmax : 1) * (nmax > 0 ? nmax : 1) * sizeof (double));
  for (int s = jb->lo; s < jb->hi; s++)
  {
    int n = jb->n[s];
    memcpy (scratch, jb->A + jb->offA[s], (size_t) n * n * sizeof (double));
    if (jb->kind == 0)
      jb->status[s] = SOLVE (scratch, jb->b + jb->offv[s], n, jb->out + jb->offv[s], s);
    else
      jb->status[s] = INVERT (scratch, jb->out + jb->offA[s], n);
  }
  free (scratch);
  return NULL;
}

static int
run_batch (int kind, int nsys, const int *n, const int64_t *offA, const double *A,
           const int64_t *offv, const double *b, double *out, int *status, int nthreads)
{
  PREPARE ();
  if (nthreads < 1)
    nthreads = 1;
  if (nthreads > nsys)
    nthreads = nsys > 0 ? nsys : 1;
  pthread_t *tid = (pthread_t *) malloc (sizeof (pthread_t) * nthreads);
  job_t *jobs = (job_t *) malloc (sizeof (job_t) * nthreads);
  for (int t = 0; t < nthreads; t++)
  {
    jobs[t].kind = kind;
    jobs[t].lo = (int) ((int64_t) nsys * t / nthreads);
    jobs[t].hi = (int) ((int64_t) nsys * (t + 1) / nthreads);
    jobs[t].n = n;
    jobs[t].offA = offA;
    jobs[t].A = A;
    jobs[t].offv = offv;
    jobs[t].b = b;
    jobs[t].out = out;
    jobs[t].status = status;
  }
  for (int t = 1; t < nthreads; t++)
    pthread_create (&tid[t], NULL, run_job, &jobs[t]);
  run_job (&jobs[0]);
  for (int t = 1; t < nthreads; t++)
    pthread_join (tid[t], NULL);
  free (tid);
  free (jobs);
  return 0;
}

/* Solve A_s x_s = b_s for every system s.  A is read-only here (copied per
   call); x receives the solution at offv[s]; status[s] the reference code. */
int
EXPORT (batch_solve) (int nsys, const int *n, const int64_t *offA, const double *A,
                      const int64_t *offv, const double *b, double *x, int *status, int nthreads)
{
  return run_batch (0, nsys, n, offA, A, offv, b, x, status, nthreads);
}

/* Invert every A_s into inv at offA[s]; status[s] the reference code. */
int
EXPORT (batch_invert) (int nsys, const int *n, const int64_t *offA, const double *A,
                       double *inv, int *status, int nthreads)
{
  return run_batch (1, nsys, n, offA, A, NULL, NULL, inv, status, nthreads);
}

const char *
EXPORT (error_string) (int code)
{
  return ERRSTR (code);
}
