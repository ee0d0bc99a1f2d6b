// Shared device-side definitions of the batched dense-solve engine.
//
// Arithmetic contract of the FP64 ("exact") kernels: the LU factorisation of
// every system reproduces, bit for bit, the factorisation that the reference's
// GSL build computes (software/gsl-2.6/linalg/lu.c:62-288 with the CBLAS loops
// of cblas/source_{ger,gemm,trsm,iamax}_r.h):
//   * pivot of column j: first row, in current row order, with the strictly
//     largest |a_ij| over rows not yet pivoted; NaN never wins; an all-zero
//     column keeps the row at position j (cblas idamax);
//   * multipliers l = a * fl(1/u_jj) when |u_jj| >= DBL_MIN, else a / u_jj
//     (lu.c:162-176);
//   * every Schur-complement entry is updated as fl(a - fl(l * u)), one k at a
//     time in increasing k, with no fused multiply-add.
// The __dmul_rn / __dsub_rn intrinsics are never contracted by nvcc, which is
// what keeps the updates unfused.  Rows never move in registers; each row
// carries its current position so that ties break exactly as GSL's physical
// row swaps would.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ss {

// Return codes of the reference (source/matrix_cpu.c:59-72, 145, 175, 183;
// GSL_EDOM = 1 from lu.c:311/345/449).
constexpr int kOk = 0;
constexpr int kResidRel = 2;
constexpr int kResidAbs = 3;
constexpr int kSolveSingular = 4;
constexpr int kInvertSingular = 1;
// GSL_ESING: invert_matrix's code when U has an infinite pivot.  LU_invx
// (lu.c:458-463) inverts U in place, leaving 1/u_jj = 0 on the diagonal, and
// gsl_linalg_tri_invert refuses the unit lower triangle for that zero
// (invtri.c:233-245).  The output is left untouched.
constexpr int kInvertInfPivot = 21;
// Engine status (not a reference code): a kernel's bounded wait for its own
// staging copy ran out, so the system was not processed.  No correct run
// produces it; it exists so that a stalled copy ends the kernel instead of
// hanging the GPU.
constexpr int kStageTimeout = -3;

// residual threshold of cpu_solve_matrix (reference source/python.h:98)
constexpr double kResidEps = 1.0e-6;
constexpr double kDblMin = 2.2250738585072014e-308;

// Per-system diagnostic bits written to the optional diag array.
constexpr int kDiagExact = 1 << 8;        // result produced by the GSL-exact FP64 path
constexpr int kDiagFallback = kDiagExact; // (mixed mode: the refinement did not accept it)
constexpr int kDiagNoConverge = 1 << 9;   // refinement stalled (reason for fallback)
constexpr int kDiagIllCond = 1 << 10;     // condition estimate above threshold
constexpr int kDiagIterMask = 0xff;       // refinement iterations used

enum Kind : int { kSolve = 0, kInvert = 1 };

// One launch's view of a batch.  All pointers are device pointers.
struct BatchView {
  const int* n;           // [nsys] order of each system
  const int64_t* offA;    // [nsys] element offset of A_s (and of its inverse)
  const int64_t* offv;    // [nsys] element offset of b_s and x_s (solve only)
  const double* A;        // packed row-major matrices
  const double* b;        // packed right-hand sides (solve only)
  double* out;            // x (solve) or A^-1 (invert), same packing
  int* status;            // [nsys] reference return code per system
  int* diag;              // [nsys] diagnostic bits, may be null
  const int* list;        // systems of this bucket, indices into the batch
  int count;              // number of systems in list
  const int* count_dev = nullptr;   // if set, the number of systems in list is read here
                                    // (a list filled on the device by an earlier launch)
};

// Number of systems a launch serves: the device-side count when the list was
// filled on the device, else the host-side count.
__device__ __forceinline__ int batch_count(const BatchView& bv) {
  return bv.count_dev ? *bv.count_dev : bv.count;
}

// Mixed-precision tuning (per launch).
struct MixedParams {
  int max_iter;           // refinement iterations before declaring a stall
  double tol;             // stop when max|dx| <= tol * max|x|
  double cond_limit;      // condition estimate above which exact FP64 is used
  double resid_margin;    // residual-check value above which exact FP64 decides the code
};

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// GSL multiplier rule (lu.c:162-176).  The division only runs for a pivot
// below DBL_MIN; the test is the same for every lane of a step.
__device__ __forceinline__ double gsl_multiplier(double a, double ujj, double rinv) {
  if (fabs(ujj) >= kDblMin) return mul_rn(a, rinv);
  return div_rn(a, ujj);
}

// Pivot key: |a| with NaN mapped to 0 (never strictly greater than the running
// maximum in cblas idamax).  Rows that cannot be chosen use -1.
__device__ __forceinline__ double pivot_key(double a) {
  double v = fabs(a);
  return (v == v) ? v : 0.0;
}

// (key, pos) ordering of the pivot search: larger key wins, ties go to the
// smaller current position (first index in GSL's row order).
__device__ __forceinline__ bool pivot_better(double k1, int p1, double k2, int p2) {
  return (k1 > k2) || (k1 == k2 && p1 < p2);
}

}  // namespace ss
