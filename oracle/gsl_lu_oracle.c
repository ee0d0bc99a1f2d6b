/*
 * CPU ORACLE -- test infrastructure only.
 *
 * A plain-C restatement of the arithmetic behind the reference's GSL build of
 * solve_matrix / invert_matrix (source/matrix_cpu.c), which calls the vendored
 * GSL 2.6 LU routines (software/gsl-2.6/linalg/lu.c, invtri.c, trimult.c) and
 * the reference CBLAS loops (software/gsl-2.6/cblas/source_*.h).  It exists so
 * that the tests, smoke() and the bench's CPU-baseline leg can check the CUDA
 * engine; the engine itself never calls, links or loads anything in this file.
 *
 * Parity pin: the tests compare this restatement with (a) the reference's own
 * matrix_cpu.c + vendored GSL compiled from source into oracle/_ref/ by
 * oracle/Makefile, and (b) the reference's unit-test fixtures
 * (source/tests/test_data/matrix/*, converted into tests/golden/).
 *
 * Why the factorisation is bit-identical to GSL's recursive LU_decomp_L3:
 *   every entry of the Schur complement receives its updates
 *       a <- fl(a - fl(l * u))
 *   one k at a time, in increasing k, whether the update is issued by
 *   dger (LU_decomp_L2, lu.c:185), dtrsm (lu.c:266, source_trsm_r.h Left/Lower/
 *   NoTrans loop) or dgemm (lu.c:269, source_gemm_r.h k-outer loop); the pivot of
 *   column j is chosen only after all k < j updates reached that column; the
 *   multipliers are l = a * fl(1/ajj) when |ajj| >= DBL_MIN and a / ajj
 *   otherwise (lu.c:162-176).  A right-looking unblocked loop with the same
 *   per-entry order therefore yields the same bits for finite input (the only
 *   difference is dgemm skipping exact-zero multipliers, which can change the
 *   sign of a zero but never a comparison).  The file is compiled with
 *   -ffp-contract=off so that no multiply-add is fused.
 *
 * The inverse (lu.c:415-481) is restated with unblocked triangular inverses and
 * an unblocked U^-1 L^-1 product; for n > 24 GSL groups those sums
 * recursively, so the inverse matches GSL to rounding, not bit for bit.  The
 * singular test that decides invert_matrix's return code depends only on the
 * factorisation and is exact.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* GSL's EPSILON-style residual threshold used by cpu_solve_matrix
   (reference source/python.h:98, EPSILON = 1.e-6). */
#define ORACLE_RESID_EPS 1.0e-6

/* GSL_EDOM, returned by LU_svx / LU_invx on an exactly singular U
   (gsl_errno.h: GSL_EDOM = 1). */
#define ORACLE_GSL_EDOM 1

/* GSL_ESING (gsl_errno.h: 21), returned by gsl_linalg_tri_invert when the
   triangle it is given has an exact zero on its diagonal (invtri.c:233-245). */
#define ORACLE_GSL_ESING 21

/* First index of the strict maximum of |a[i*n+j]| over i in [j, n), scanning
   from max = 0.0 like cblas idamax (cblas/source_iamax_r.h): NaNs are never
   chosen and an all-zero column returns j. */
static int
pivot_row (const double *a, int n, int j)
{
  double best = 0.0;
  int r = j;
  for (int i = j; i < n; i++)
  {
    double v = fabs (a[(size_t) i * n + j]);
    if (v > best)
    {
      best = v;
      r = i;
    }
  }
  return r;
}

/* PA = LU in place (lu.c:62 gsl_linalg_LU_decomp).  ipiv[j] is the row swapped
   with row j at step j; perm[i] is the original row now at row i (the
   gsl_permutation built at lu.c:95-109).  Returns the permutation sign. */
int
oracle_lu_decomp (double *a, int n, int *ipiv, int *perm)
{
  for (int j = 0; j < n; j++)
  {
    int p = pivot_row (a, n, j);
    ipiv[j] = p;
    if (p != j)
    {
      double *rj = a + (size_t) j * n, *rp = a + (size_t) p * n;
      for (int k = 0; k < n; k++)
      {
        double t = rj[k];
        rj[k] = rp[k];
        rp[k] = t;
      }
    }
    if (j < n - 1)
    {
      double ajj = a[(size_t) j * n + j];
      if (fabs (ajj) >= DBL_MIN)
      {
        double r = 1.0 / ajj;
        for (int i = j + 1; i < n; i++)
          a[(size_t) i * n + j] *= r;
      }
      else
      {
        for (int i = j + 1; i < n; i++)
          a[(size_t) i * n + j] /= ajj;
      }
      for (int i = j + 1; i < n; i++)
      {
        double l = a[(size_t) i * n + j];
        double *ri = a + (size_t) i * n;
        const double *rj = a + (size_t) j * n;
        for (int k = j + 1; k < n; k++)
        {
          double prod = l * rj[k];
          ri[k] = ri[k] - prod;
        }
      }
    }
  }
  int sign = 1;
  for (int i = 0; i < n; i++)
    perm[i] = i;
  for (int i = 0; i < n; i++)
  {
    int q = ipiv[i];
    if (perm[q] != perm[i])
    {
      int t = perm[q];
      perm[q] = perm[i];
      perm[i] = t;
      sign = -sign;
    }
  }
  return sign;
}

/* lu.c:540 singular(): exact zero on the diagonal of U. */
int
oracle_lu_singular (const double *lu, int n)
{
  for (int i = 0; i < n; i++)
    if (lu[(size_t) i * n + i] == 0.0)
      return 1;
  return 0;
}

/* lu.c:291 gsl_linalg_LU_solve -> lu.c:329 LU_svx: x = P b, then the two
   row-oriented dtrsv loops of cblas/source_trsv_r.h (forward: ascending j;
   backward: i descending, inner j ascending from i+1, division by U_ii). */
int
oracle_lu_solve (const double *lu, int n, const int *perm, const double *b, double *x)
{
  if (oracle_lu_singular (lu, n))
    return ORACLE_GSL_EDOM;
  for (int i = 0; i < n; i++)
    x[i] = b[perm[i]];
  for (int i = 1; i < n; i++)
  {
    double t = x[i];
    const double *row = lu + (size_t) i * n;
    for (int j = 0; j < i; j++)
    {
      double prod = row[j] * x[j];
      t = t - prod;
    }
    x[i] = t;
  }
  x[n - 1] = x[n - 1] / lu[(size_t) (n - 1) * n + (n - 1)];
  for (int i = n - 2; i >= 0; i--)
  {
    double t = x[i];
    const double *row = lu + (size_t) i * n;
    for (int j = i + 1; j < n; j++)
    {
      double prod = row[j] * x[j];
      t = t - prod;
    }
    x[i] = t / row[i];
  }
  return 0;
}

/* The residual check of cpu_solve_matrix (matrix_cpu.c:155-187): y = A x by
   the row-major dgemv loop (cblas/source_gemv_r.h, ascending j), then the
   first failing row decides: b_i > 0 and |(y_i - b_i)/y_i| > 1e-6 -> 2,
   otherwise |y_i - b_i| > 1e-6 -> 3. */
int
oracle_residual_code (const double *a, const double *b, const double *x, int n)
{
  for (int i = 0; i < n; i++)
  {
    double t = 0.0;
    const double *row = a + (size_t) i * n;
    for (int j = 0; j < n; j++)
    {
      double prod = row[j] * x[j];
      t = t + prod;
    }
    double y = 0.0 + 1.0 * t;
    if (b[i] > 0.0)
    {
      if (fabs ((y - b[i]) / y) > ORACLE_RESID_EPS)
        return 2;
    }
    else if (fabs (y - b[i]) > ORACLE_RESID_EPS)
      return 3;
  }
  return 0;
}

/* matrix_cpu.c:97 cpu_solve_matrix.  a is overwritten by its LU factors, as in
   the reference.  Returns 0, 2, 3 or 4; x is written unless the code is 4. */
int
oracle_solve_matrix (double *a, const double *b, int n, double *x)
{
  if (n <= 0)
    return 4;
  size_t nn = (size_t) n * n;
  double *copy = (double *) malloc (nn * sizeof (double));
  double *sol = (double *) malloc ((size_t) n * sizeof (double));
  int *ipiv = (int *) malloc ((size_t) n * sizeof (int));
  int *perm = (int *) malloc ((size_t) n * sizeof (int));
  int code;
  memcpy (copy, a, nn * sizeof (double));
  oracle_lu_decomp (a, n, ipiv, perm);
  if (oracle_lu_solve (a, n, perm, b, sol))
    code = 4;
  else
  {
    code = oracle_residual_code (copy, b, sol, n);
    memcpy (x, sol, (size_t) n * sizeof (double));
  }
  free (copy);
  free (sol);
  free (ipiv);
  free (perm);
  return code;
}

/* In-place inverse of an upper, non-unit triangle (LAPACK dtrti2 order, which
   GSL's triangular_inverse_L2 follows for n <= 24, invtri.c). */
static void
upper_inverse (double *u, int n)
{
  for (int i = 0; i < n; i++)
  {
    u[(size_t) i * n + i] = 1.0 / u[(size_t) i * n + i];
    double aii = -u[(size_t) i * n + i];
    /* v = Uinv[0:i,0:i] * U[0:i, i] (dtrmv upper, no-trans), then v *= aii */
    for (int r = 0; r < i; r++)
    {
      double t = 0.0;
      for (int c = r; c < i; c++)
        t += u[(size_t) r * n + c] * u[(size_t) c * n + i];
      u[(size_t) r * n + i] = t;
    }
    for (int r = 0; r < i; r++)
      u[(size_t) r * n + i] *= aii;
  }
}

/* In-place inverse of a unit lower triangle (invtri.c lower branch). */
static void
unit_lower_inverse (double *l, int n)
{
  for (int jj = 0; jj < n; jj++)
  {
    int j = n - 1 - jj;
    for (int r = n - 1; r > j; r--)
    {
      double t = l[(size_t) r * n + j];
      for (int c = j + 1; c < r; c++)
        t += l[(size_t) r * n + c] * l[(size_t) c * n + j];
      l[(size_t) r * n + j] = t;
    }
    for (int r = j + 1; r < n; r++)
      l[(size_t) r * n + j] = -l[(size_t) r * n + j];
  }
}

/* matrix_cpu.c:224 cpu_invert_matrix -> lu.c:415 gsl_linalg_LU_invert.
   Returns 0, or GSL_EDOM (1) when U has an exact zero on its diagonal, or
   GSL_ESING (21) when U has an infinite one, in which cases inv is left
   untouched as in the reference.  The second code comes from the order of
   LU_invx (lu.c:458-463): U is inverted in place first, which leaves 1/u_ii on
   the diagonal, and gsl_linalg_tri_invert then checks that diagonal for exact
   zeros before it inverts the unit lower triangle; 1/(+-Inf) is zero. */
int
oracle_invert_matrix (double *a, double *inv, int n)
{
  if (n <= 0)
    return ORACLE_GSL_EDOM;
  size_t nn = (size_t) n * n;
  int *ipiv = (int *) malloc ((size_t) n * sizeof (int));
  int *perm = (int *) malloc ((size_t) n * sizeof (int));
  oracle_lu_decomp (a, n, ipiv, perm);
  if (oracle_lu_singular (a, n))
  {
    free (ipiv);
    free (perm);
    return ORACLE_GSL_EDOM;
  }
  for (int i = 0; i < n; i++)
    if (1.0 / a[(size_t) i * n + i] == 0.0)
    {
      free (ipiv);
      free (perm);
      return ORACLE_GSL_ESING;
    }
  double *w = (double *) malloc (nn * sizeof (double));
  double *x = (double *) malloc (nn * sizeof (double));
  memcpy (w, a, nn * sizeof (double));
  upper_inverse (w, n);
  unit_lower_inverse (w, n);
  /* X = Uinv * Linv (trimult.c gsl_linalg_tri_UL): X[i][k] = sum over
     m >= max(i,k) of Uinv[i][m] * Linv[m][k], with Linv[m][m] = 1. */
  for (int i = 0; i < n; i++)
    for (int k = 0; k < n; k++)
    {
      int m0 = i > k ? i : k;
      double t = 0.0;
      for (int m = m0; m < n; m++)
      {
        double lmk = (m == k) ? 1.0 : w[(size_t) m * n + k];
        t += w[(size_t) i * n + m] * lmk;
      }
      x[(size_t) i * n + k] = t;
    }
  /* lu.c:473-477: gsl_permute_vector_inverse on every row: out[i][perm[j]] = X[i][j] */
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      inv[(size_t) i * n + perm[j]] = x[(size_t) i * n + j];
  free (w);
  free (x);
  free (ipiv);
  free (perm);
  return 0;
}

/* matrix_cpu.c:59 cpu_matrix_error_string. */
const char *
oracle_matrix_error_string (int code)
{
  switch (code)
  {
  case 2:
    return "some matrix rows failing relative error check";
  case 3:
    return "some matrix rows failing absolute error check";
  case 4:
    return "Unsolvable matrix! Determinant is zero. Defaulting to no change";
  default:
    return "bad return from solve_matrix";
  }
}
