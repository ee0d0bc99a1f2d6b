// Sub-warp-per-system kernels for n <= 32 (ion-balance systems, n = 2..27 in
// practice, and small macro atoms).
//
// A group of G lanes (G in {4, 8, 16, 32}, so 8/4/2/1 systems per warp) owns
// one system; lane r holds row r of A in registers (NP doubles, NP >= n, all
// indices compile-time after unrolling).  Rows never move: each carries its
// current position `pos`, the pivot search is three redux.sync reductions of
// (|a| bits, position) over the group, and the pivot row is broadcast through a
// small shared buffer.
//
// solve  : GSL-exact LU (lu.c:62-288), then the two row-oriented triangular
//          sweeps of LU_svx (lu.c:329-360, cblas/source_trsv_r.h) in GSL's
//          operation order, then the reference residual check
//          (matrix_cpu.c:155-187) on the original A held in shared memory.
// invert : in-place Gauss-Jordan whose below-pivot updates are the GSL-exact
//          LU updates (so the pivots, U and the singular test of lu.c:540 are
//          GSL's), above-pivot and already-inverted columns eliminated in the
//          same sweep; columns are unscrambled in reverse pivot order at the end.
#pragma once
#include "ss_common.cuh"

namespace ss {

constexpr int kSmallThreads = 128;

template <int NP>
struct SmallSmem {
  static constexpr int S = NP + 1;   // odd row stride (in doubles) avoids bank conflicts
  double stage[NP * S];              // A as loaded (solve: kept for the residual check)
  double piv[NP];                    // broadcast pivot row
  double xs[NP];                     // solution in natural order
  float fpiv[NP];                    // broadcast pivot row (mixed path)
  double rsc[NP];                    // row scales (mixed path)
  double csc[NP];                    // column scales (mixed path)
  int ipiv[NP];                      // position swapped with j at step j
  int lop[NP];                       // lane holding position i
  int csrc[NP];                      // column unscramble map (invert)
};

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  const int wlane = threadIdx.x & 31;
  return (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (wlane & ~(G - 1)));
}

// Coalesced load of system s into sm.stage, every load of the lane issued
// before the first shared-memory store so they are all in flight together.
template <int NP, int G>
__device__ __forceinline__ void small_stage(SmallSmem<NP>& sm, const double* __restrict__ Ag, int n, int lane,
                                            unsigned gmask) {
  constexpr int S = SmallSmem<NP>::S;
  constexpr int PER = (NP * NP + G - 1) / G;
  const int nn = n * n;
  double v[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = lane + u * G;
    v[u] = (e < nn) ? __ldg(Ag + e) : 0.0;
  }
  // element e = r * n + c; track (r, c) incrementally instead of dividing
  int r = lane / n, c = lane - (lane / n) * n;
  const int dr = G / n, dc = G - (G / n) * n;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    if (lane + u * G < nn) sm.stage[r * S + c] = v[u];
    r += dr;
    c += dc;
    if (c >= n) { c -= n; ++r; }
  }
  __syncwarp(gmask);
}

// GSL-exact factorisation (KIND == kSolve: LU; kInvert: Gauss-Jordan) of the
// row held in a[].  Returns true when U has an exact zero on its diagonal.
template <int KIND, int NP, int G>
__device__ __forceinline__ bool small_exact_factor(SmallSmem<NP>& sm, double (&a)[NP], int n, int lane,
                                                   unsigned gmask, int& pos, bool& inf_piv) {
  const bool act = lane < n;
  bool done = false;
  bool sing = false;
  inf_piv = false;
  pos = lane;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    if (j < n && !sing) {
      // first strict maximum of |a| in current row order (cblas idamax): the
      // eligible rows' keys carry bit 63 and NaN counts as zero; ties go to the
      // smaller position
      const bool elig = act && !done;
      unsigned long long key = 0ull;
      if (elig) {
        const double v = fabs(a[j]);
        key = (v == v) ? (static_cast<unsigned long long>(__double_as_longlong(v)) | (1ull << 63)) : (1ull << 63);
      }
      const unsigned hi = unsigned(key >> 32), lo = unsigned(key);
      const unsigned mh = __reduce_max_sync(gmask, hi);
      const unsigned ml = __reduce_max_sync(gmask, hi == mh ? lo : 0u);
      const int kp = int(__reduce_min_sync(gmask, (elig && hi == mh && lo == ml) ? unsigned(pos) : 0xffffffffu));
      const int p = (__ffs(__ballot_sync(gmask, elig && pos == kp)) - 1) & (G - 1);
      const bool was_done = done;
      if (lane == p) {
        pos = j;
        done = true;
      } else if (pos == j) {
        pos = kp;
      }
      if (lane == 0) sm.ipiv[j] = kp;
      if (lane == p) {
#pragma unroll
        for (int k = (KIND == kSolve ? j : 0); k < NP; ++k) sm.piv[k] = a[k];
      }
      __syncwarp(gmask);
      const double ujj = sm.piv[j];
      inf_piv |= isinf(ujj);
      if (ujj == 0.0) {
        sing = true;   // lu.c:540 singular(): the result is decided
      } else {
        const double rinv = __drcp_rn(ujj);   // correctly rounded, = fl(1/ujj)
        if (KIND == kSolve) {
          if (act && !was_done && lane != p) {
            const double l = gsl_multiplier(a[j], ujj, rinv);
            a[j] = l;
#pragma unroll
            for (int k = j + 1; k < NP; ++k) a[k] = sub_rn(a[k], mul_rn(l, sm.piv[k]));
          }
        } else {
          if (lane == p) {
#pragma unroll
            for (int k = 0; k < NP; ++k) a[k] = (k == j) ? rinv : mul_rn(a[k], rinv);
          } else if (act) {
            const double l = was_done ? mul_rn(a[j], rinv) : gsl_multiplier(a[j], ujj, rinv);
#pragma unroll
            for (int k = 0; k < NP; ++k)
              if (k != j) a[k] = sub_rn(a[k], mul_rn(l, sm.piv[k]));
            a[j] = -l;
          }
        }
      }
      __syncwarp(gmask);
    }
  }
  return sing;
}

// Reference residual check of x (sm.xs, natural order) against the original
// A (sm.stage); the first failing row decides (matrix_cpu.c:162-187).  Also
// returns, in *worst, the largest check value over all rows.
template <int NP, int G>
__device__ __forceinline__ int small_residual_code(SmallSmem<NP>& sm, const double* __restrict__ Ag,
                                                   const double* __restrict__ bg, int n, int lane, unsigned gmask,
                                                   double* worst) {
  int code = 0;
  double chk = 0.0;
  if (lane < n) {
    double acc = 0.0;
    const double* __restrict__ arow = Ag + lane * n;
#pragma unroll
    for (int k = 0; k < NP; ++k)
      if (k < n) acc = add_rn(acc, mul_rn(__ldg(arow + k), sm.xs[k]));
    const double y = add_rn(0.0, acc);
    const double bi = bg[lane];
    if (bi > 0.0) {
      chk = fabs(div_rn(sub_rn(y, bi), y));
      if (chk > kResidEps) code = kResidRel;
    } else {
      chk = fabs(sub_rn(y, bi));
      if (chk > kResidEps) code = kResidAbs;
    }
    if (!(chk == chk)) chk = 1.0e300;   // a NaN check value passes the reference test; flag it
  }
  int first = code ? lane : 0x7fffffff;
  int fcode = code;
#pragma unroll
  for (int off = G / 2; off > 0; off >>= 1) {
    const int of = __shfl_xor_sync(gmask, first, off, G);
    const int oc = __shfl_xor_sync(gmask, fcode, off, G);
    const double ow = __shfl_xor_sync(gmask, chk, off, G);
    if (of < first) { first = of; fcode = oc; }
    chk = fmax(chk, ow);
  }
  *worst = chk;
  return fcode;
}

// Complete GSL-exact solve of the staged system (Ag: the same matrix in global
// memory, for the residual check); writes x and returns the code.  The staged
// copy is overwritten with the factors.
template <int NP, int G>
__device__ __forceinline__ int small_exact_solve(SmallSmem<NP>& sm, const double* __restrict__ Ag,
                                                 const double* __restrict__ bg, double* __restrict__ xg, int n,
                                                 int lane, unsigned gmask) {
  constexpr int S = SmallSmem<NP>::S;
  const bool act = lane < n;
  double a[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) a[k] = (act && k < n) ? sm.stage[lane * S + k] : 0.0;
  int pos;
  bool inf_piv;
  if (small_exact_factor<kSolve, NP, G>(sm, a, n, lane, gmask, pos, inf_piv)) return kSolveSingular;
  if (act) sm.lop[pos] = lane;
  double t = act ? bg[lane] : 0.0;   // (P b) at this row's position
  __syncwarp(gmask);
  // forward sweep with unit L: every entry takes its updates in ascending j
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    if (j < n) {
      const double yj = __shfl_sync(gmask, t, sm.lop[j], G);
      if (act && pos > j) t = sub_rn(t, mul_rn(a[j], yj));
    }
  }
  // backward sweep, row-oriented: x_i = (y_i - sum_{k>i} U_ik x_k) / U_ii; the
  // rows of U go to shared memory by position and one lane walks them
  if (act) {
#pragma unroll
    for (int k = 0; k < NP; ++k) sm.stage[pos * S + k] = a[k];
    sm.piv[pos] = t;
  }
  __syncwarp(gmask);
  if (lane == 0) {
    for (int i = n - 1; i >= 0; --i) {
      const double* __restrict__ urow = &sm.stage[i * S];
      double u = sm.piv[i];
#pragma unroll 4
      for (int k = i + 1; k < n; ++k) u = sub_rn(u, mul_rn(urow[k], sm.xs[k]));
      sm.xs[i] = div_rn(u, urow[i]);
    }
  }
  __syncwarp(gmask);
  double worst;
  const int code = small_residual_code<NP, G>(sm, Ag, bg, n, lane, gmask, &worst);
  for (int k = lane; k < n; k += G) xg[k] = sm.xs[k];
  return code;
}

template <int KIND, int NP, int G>
__global__ void __launch_bounds__(kSmallThreads)
small_exact_kernel(BatchView bv) {
  static_assert(G == 4 || G == 8 || G == 16 || G == 32, "group size");
  static_assert(NP <= G, "one row per lane");
  constexpr int GPB = kSmallThreads / G;       // groups per block
  constexpr int S = SmallSmem<NP>::S;
  __shared__ __align__(16) SmallSmem<NP> smem_all[GPB];

  const int grp = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  const unsigned gmask = group_mask<G>();
  SmallSmem<NP>& sm = smem_all[grp];

  const int count = batch_count(bv);
  for (int item = blockIdx.x * GPB + grp; item < count; item += gridDim.x * GPB) {
    const int s = bv.list[item];
    const int n = bv.n[s];
    small_stage<NP, G>(sm, bv.A + bv.offA[s], n, lane, gmask);

    if (KIND == kSolve) {
      const int64_t ov = bv.offv[s];
      const int code = small_exact_solve<NP, G>(sm, bv.A + bv.offA[s], bv.b + ov, bv.out + ov, n, lane, gmask);
      if (lane == 0) {
        bv.status[s] = code;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
    } else {
      const bool act = lane < n;
      double a[NP];
#pragma unroll
      for (int k = 0; k < NP; ++k) a[k] = (act && k < n) ? sm.stage[lane * S + k] : 0.0;
      int pos;
      bool inf_piv;
      const bool sing = small_exact_factor<kInvert, NP, G>(sm, a, n, lane, gmask, pos, inf_piv);
      // GSL's LU_invx inverts U in place and then finds 1/u_jj = 0 on the
      // diagonal for an infinite pivot: GSL_ESING, output untouched
      const int code = sing ? kInvertSingular : (inf_piv ? kInvertInfPivot : kOk);
      if (code == kOk) {
        // rows of W by position, then the reverse-order column unscramble
        if (act) {
#pragma unroll
          for (int k = 0; k < NP; ++k)
            if (k < n) sm.stage[pos * S + k] = a[k];
        }
        if (lane == 0) {
          for (int c = 0; c < n; ++c) sm.csrc[c] = c;
          for (int j = n - 1; j >= 0; --j) {
            const int q = sm.ipiv[j];
            if (q != j) {
              const int tt = sm.csrc[j];
              sm.csrc[j] = sm.csrc[q];
              sm.csrc[q] = tt;
            }
          }
        }
        __syncwarp(gmask);
        double* __restrict__ Og = bv.out + bv.offA[s];
        for (int e = lane; e < n * n; e += G) {
          const int r = e / n;
          Og[e] = sm.stage[r * S + sm.csrc[e - r * n]];
        }
      }
      if (lane == 0) {
        bv.status[s] = code;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
    }
    __syncwarp(gmask);
  }
}

}  // namespace ss
