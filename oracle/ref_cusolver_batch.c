/*
 * Reference-arm helper -- measurement infrastructure only, never on the engine's path.
 *
 * Serial batch loop around the reference's own cuSOLVER build
 * (source/matrix_gpu.cu: gpu_solve_matrix :264-307, gpu_invert_matrix
 * :332-384), compiled unmodified from the reference tree by oracle/Makefile
 * into oracle/_ref/libref_cusolver.so.  Each system is one call, exactly as the
 * reference's CUDA_ON build calls it once per cell through solve_matrix /
 * invert_matrix (source/matrix_cpu.c:310-349): every call allocates, copies,
 * factorises with cusolverDnDgetrf/getrs, copies back and frees.  A is copied
 * into a scratch buffer first so the caller's batch stays intact.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int cusolver_create (void);
int cusolver_destroy (void);
int gpu_solve_matrix (double *a_matrix, double *b_vector, int size, double *x_vector);
int gpu_invert_matrix (double *matrix, double *inverse, int num_rows);

int
refgpu_create (void)
{
  return cusolver_create ();
}

int
refgpu_destroy (void)
{
  return cusolver_destroy ();
}

static int
max_order (int nsys, const int *n)
{
  int m = 1;
  for (int s = 0; s < nsys; ++s)
    if (n[s] > m)
      m = n[s];
  return m;
}

int
refgpu_batch_solve (int nsys, const int *n, const int64_t *offA, const double *A, const int64_t *offv,
                    const double *b, double *x, int *status)
{
  const size_t m = (size_t) max_order (nsys, n);
  double *a = malloc (m * m * sizeof (double));
  double *bb = malloc (m * sizeof (double));
  if (!a || !bb)
  {
    free (a);
    free (bb);
    return -1;
  }
  for (int s = 0; s < nsys; ++s)
  {
    const size_t ns = (size_t) n[s];
    memcpy (a, A + offA[s], ns * ns * sizeof (double));
    memcpy (bb, b + offv[s], ns * sizeof (double));
    status[s] = gpu_solve_matrix (a, bb, n[s], x + offv[s]);
  }
  free (a);
  free (bb);
  return 0;
}

int
refgpu_batch_invert (int nsys, const int *n, const int64_t *offA, const double *A, double *Ainv, int *status)
{
  const size_t m = (size_t) max_order (nsys, n);
  double *a = malloc (m * m * sizeof (double));
  if (!a)
    return -1;
  for (int s = 0; s < nsys; ++s)
  {
    const size_t ns = (size_t) n[s];
    memcpy (a, A + offA[s], ns * ns * sizeof (double));
    status[s] = gpu_invert_matrix (a, Ainv + offA[s], n[s]);
  }
  free (a);
  return 0;
}
