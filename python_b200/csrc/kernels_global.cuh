// CTA-per-system kernels for n > 128 (large macro atoms, full ion matrices).
//
// The system is factorised in a global-memory workspace W (the output buffer
// for an inverse, a per-CTA scratch slab for a solve), panel by panel:
//   1. the n x NB panel is staged in shared memory and factorised there with
//      physical row swaps (first strict maximum, as GSL's idamax), recording
//      the multipliers M (n x NB) of every row at every panel step;
//   2. the remaining columns are processed in CW-wide chunks: the panel's row
//      swaps are applied (lu.c:263 apply_pivots), the pivot rows' values at
//      their own step are rebuilt by the unit-lower recurrence
//      V_k = W_k - sum_{k'<k} M[k][k'] V_k' (the dtrsm of lu.c:266), and every
//      other row takes W_r -= sum_k M[r][k] V_k with one rounding per product
//      and per difference, k ascending (the dgemm of lu.c:269).
// Each entry of the LU region therefore sees exactly GSL's sequence of
// operations.  For an inverse the same sweep also eliminates the rows above
// the pivots and the already-inverted columns (blocked Gauss-Jordan), the
// pivot rows are scaled by 1/u_kk, and the columns are unscrambled at the end.
#pragma once
#include "ss_common.cuh"

namespace ss {

constexpr int kGThreads = 256;
constexpr int kGNB = 8;       // panel width
constexpr int kGCW = 64;      // column chunk of the deferred update
constexpr int kGPS = kGNB + 1; // shared-memory row stride of the panel (odd: no bank conflicts)

__host__ __device__ constexpr size_t global_smem_bytes(int nmax) {
  return size_t(2) * nmax * kGPS * sizeof(double)      // panel + multipliers
       + size_t(kGNB) * kGCW * sizeof(double)          // V chunk
       + size_t(nmax) * sizeof(int)                    // pivots
       + size_t(nmax) * sizeof(int)                    // column map
       + size_t(32) * sizeof(double);                  // per-step scalars
}

// DIRECT = true is the variant behind solve_matrix_batched_noalloc: system
// `item` is batch entry `item` (no bucket list) and a system larger than nmax
// is refused with status -1 instead of being factorised.
template <int KIND, bool DIRECT = false>
__global__ void __launch_bounds__(kGThreads, 1)
global_exact_kernel(BatchView bv, int nmax, double* scratch, int64_t slab) {
  extern __shared__ __align__(16) double gsm[];
  double* Ps = gsm;                                   // [nmax][PS]
  double* Ms = Ps + size_t(nmax) * kGPS;              // [nmax][PS]
  double* Vs = Ms + size_t(nmax) * kGPS;              // [NB][CW]
  double* rinv_s = Vs + kGNB * kGCW;                  // [NB]
  double* red_k = rinv_s + kGNB;                      // [8] warp keys
  int* ipiv = reinterpret_cast<int*>(rinv_s + 32);    // [nmax]
  int* cmap = ipiv + nmax;                            // [nmax]
  __shared__ int red_r[kGThreads / 32];
  __shared__ int sing_s;

  const int t = threadIdx.x;
  const int wid = t >> 5, wl = t & 31;

  for (int item = blockIdx.x; item < bv.count; item += gridDim.x) {
    const int s = DIRECT ? item : bv.list[item];
    const int n = bv.n[s];
    if (DIRECT && (n < 1 || n > nmax)) {
      if (t == 0) bv.status[s] = -1;
      continue;
    }
    const double* __restrict__ Ag = bv.A + bv.offA[s];
    double* __restrict__ W = (KIND == kInvert) ? bv.out + bv.offA[s] : scratch + int64_t(blockIdx.x) * slab;
    const int64_t nn = int64_t(n) * n;
    for (int64_t e = t; e < nn; e += kGThreads) W[e] = Ag[e];
    if (t == 0) sing_s = 0;
    __syncthreads();

    bool sing = false;
    for (int j0 = 0; j0 < n && !sing; j0 += kGNB) {
      const int nb = min(kGNB, n - j0);
      // ---- 1. panel into shared memory ---------------------------------
      for (int e = t; e < n * kGNB; e += kGThreads) {
        const int r = e / kGNB, k = e - r * kGNB;
        Ps[r * kGPS + k] = (k < nb) ? W[int64_t(r) * n + j0 + k] : 0.0;
        Ms[r * kGPS + k] = 0.0;
      }
      __syncthreads();
      for (int k = 0; k < nb; ++k) {
        const int j = j0 + k;
        // pivot: first strict maximum of |P[r][k]| over rows r >= j
        double bk = -1.0;
        int br = 0x7fffffff;
        for (int r = j + t; r < n; r += kGThreads) {
          const double key = pivot_key(Ps[r * kGPS + k]);
          if (pivot_better(key, r, bk, br)) { bk = key; br = r; }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const double ok = __shfl_xor_sync(0xffffffffu, bk, off);
          const int orr = __shfl_xor_sync(0xffffffffu, br, off);
          if (pivot_better(ok, orr, bk, br)) { bk = ok; br = orr; }
        }
        if (wl == 0) { red_k[wid] = bk; red_r[wid] = br; }
        __syncthreads();
        bk = -1.0; br = 0x7fffffff;
#pragma unroll
        for (int w = 0; w < kGThreads / 32; ++w)
          if (pivot_better(red_k[w], red_r[w], bk, br)) { bk = red_k[w]; br = red_r[w]; }
        const int p = br;
        if (t == 0) ipiv[j] = p;
        if (p != j) {
          if (t < kGNB) {
            const double x = Ps[j * kGPS + t]; Ps[j * kGPS + t] = Ps[p * kGPS + t]; Ps[p * kGPS + t] = x;
          } else if (t < 2 * kGNB) {
            const int c = t - kGNB;
            const double x = Ms[j * kGPS + c]; Ms[j * kGPS + c] = Ms[p * kGPS + c]; Ms[p * kGPS + c] = x;
          }
        }
        __syncthreads();
        const double ujj = Ps[j * kGPS + k];
        if (ujj == 0.0) { sing = true; break; }
        const double rinv = __drcp_rn(ujj);   // correctly rounded, = fl(1/ujj)
        double piv[kGNB];
#pragma unroll
        for (int c = 0; c < kGNB; ++c) piv[c] = Ps[j * kGPS + c];
        __syncthreads();
        for (int r = t; r < n; r += kGThreads) {
          if (r == j) continue;
          if (KIND == kSolve && r < j) continue;
          const double v = Ps[r * kGPS + k];
          const double m = (r > j) ? gsl_multiplier(v, ujj, rinv) : mul_rn(v, rinv);
          Ms[r * kGPS + k] = m;
          if (m != 0.0) {
#pragma unroll
            for (int c = 0; c < kGNB; ++c) {
              if (c == k) continue;
              if (KIND == kSolve && c < k) continue;
              Ps[r * kGPS + c] = sub_rn(Ps[r * kGPS + c], mul_rn(m, piv[c]));
            }
          }
          Ps[r * kGPS + k] = (KIND == kInvert) ? -m : m;
        }
        if (t == 0) {
          rinv_s[k] = rinv;
          Ms[j * kGPS + k] = 0.0;
          if (KIND == kInvert) {
#pragma unroll
            for (int c = 0; c < kGNB; ++c) Ps[j * kGPS + c] = (c == k) ? rinv : mul_rn(piv[c], rinv);
          }
        }
        __syncthreads();
      }
      if (sing) break;
      for (int e = t; e < n * kGNB; e += kGThreads) {
        const int r = e / kGNB, k = e - r * kGNB;
        if (k < nb) W[int64_t(r) * n + j0 + k] = Ps[r * kGPS + k];
      }
      __syncthreads();

      // ---- 2. deferred update of the other columns, CW at a time --------
      // ranges: [0, j0) then [j0+nb, n).  For a solve the left range (L of
      // earlier panels) only takes the row swaps.
      for (int side = 0; side < 2; ++side) {
        const int lo = side == 0 ? 0 : j0 + nb;
        const int hi = side == 0 ? j0 : n;
        const bool swap_only = (KIND == kSolve) && side == 0;
        for (int cA = lo; cA < hi; cA += kGCW) {
          const int cw = min(kGCW, hi - cA);
          if (t < cw) {
            const int c = cA + t;
            for (int k = 0; k < nb; ++k) {
              const int q = ipiv[j0 + k];
              if (q != j0 + k) {
                const double x = W[int64_t(j0 + k) * n + c];
                W[int64_t(j0 + k) * n + c] = W[int64_t(q) * n + c];
                W[int64_t(q) * n + c] = x;
              }
            }
            if (!swap_only) {
              for (int k = 0; k < nb; ++k) {
                double v = W[int64_t(j0 + k) * n + c];
                for (int kk = 0; kk < k; ++kk) v = sub_rn(v, mul_rn(Ms[(j0 + k) * kGPS + kk], Vs[kk * kGCW + t]));
                Vs[k * kGCW + t] = v;
              }
            }
          }
          if (swap_only) continue;
          __syncthreads();
          const int cl = t % kGCW;
          const int rg = t / kGCW;
          constexpr int RG = kGThreads / kGCW;
          if (cl < cw) {
            const int c = cA + cl;
            const int r_begin = (KIND == kInvert) ? 0 : j0;
            for (int r = r_begin + rg; r < n; r += RG) {
              double* w = W + int64_t(r) * n + c;
              if (r >= j0 && r < j0 + nb) {
                const int k = r - j0;
                double acc = Vs[k * kGCW + cl];
                if (KIND == kInvert) {
                  acc = mul_rn(acc, rinv_s[k]);
                  for (int k2 = k + 1; k2 < nb; ++k2) {
                    const double m = Ms[r * kGPS + k2];
                    if (m != 0.0) acc = sub_rn(acc, mul_rn(m, Vs[k2 * kGCW + cl]));
                  }
                }
                *w = acc;
              } else {
                double acc = *w;
                for (int k = 0; k < nb; ++k) {
                  const double m = Ms[r * kGPS + k];
                  if (m != 0.0) acc = sub_rn(acc, mul_rn(m, Vs[k * kGCW + cl]));
                }
                *w = acc;
              }
            }
          }
          __syncthreads();
        }
      }
      __syncthreads();
    }

    if (sing) {
      if (t == 0) {
        bv.status[s] = (KIND == kSolve) ? kSolveSingular : kInvertSingular;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
      __syncthreads();
      continue;
    }

    if (KIND == kInvert) {
      // W holds the inverse with its columns permuted; unscramble in reverse pivot order
      if (t == 0) {
        for (int c = 0; c < n; ++c) cmap[c] = c;
        for (int jj = n - 1; jj >= 0; --jj) {
          const int q = ipiv[jj];
          if (q != jj) { const int x = cmap[jj]; cmap[jj] = cmap[q]; cmap[q] = x; }
        }
      }
      __syncthreads();
      double* rowbuf = Ps + size_t(wid) * nmax;       // 8 warps x n doubles fit in Ps+Ms
      for (int r = wid; r < n; r += kGThreads / 32) {
        double* w = W + int64_t(r) * n;
        for (int c = wl; c < n; c += 32) rowbuf[c] = w[c];
        __syncwarp();
        for (int c = wl; c < n; c += 32) w[c] = rowbuf[cmap[c]];
        __syncwarp();
      }
      if (t == 0) {
        bv.status[s] = kOk;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
    } else {
      double* vec = Ps;                 // y, then x (natural order), n doubles each
      double* xs = Ps + nmax;
      if (t == 0) {
        // gsl_permutation from the row swaps (lu.c:95-109): cmap[i] = original row at i
        for (int i = 0; i < n; ++i) cmap[i] = i;
        for (int i = 0; i < n; ++i) {
          const int q = ipiv[i];
          if (cmap[q] != cmap[i]) { const int x = cmap[q]; cmap[q] = cmap[i]; cmap[i] = x; }
        }
      }
      __syncthreads();
      if (wid == 0) {
        const int64_t ov = bv.offv[s];
        for (int i = wl; i < n; i += 32) vec[i] = bv.b[ov + cmap[i]];
        __syncwarp();
        for (int j = 0; j < n; ++j) {
          const double yj = vec[j];
          for (int i = j + 1 + wl; i < n; i += 32) vec[i] = sub_rn(vec[i], mul_rn(W[int64_t(i) * n + j], yj));
          __syncwarp();
        }
        if (wl == 0) {
          for (int i = n - 1; i >= 0; --i) {
            const double* __restrict__ row = W + int64_t(i) * n;
            double u = vec[i];
            for (int k = i + 1; k < n; ++k) u = sub_rn(u, mul_rn(row[k], xs[k]));
            xs[i] = div_rn(u, row[i]);
          }
        }
        __syncwarp();
        int first = 0x7fffffff, fcode = 0;
        for (int i = wl; i < n; i += 32) {
          double acc = 0.0;
          const double* __restrict__ row = Ag + int64_t(i) * n;
          for (int k = 0; k < n; ++k) acc = add_rn(acc, mul_rn(row[k], xs[k]));
          const double y = add_rn(0.0, acc);
          const double bi = bv.b[ov + i];
          int code = 0;
          if (bi > 0.0) {
            if (fabs(div_rn(sub_rn(y, bi), y)) > kResidEps) code = kResidRel;
          } else if (fabs(sub_rn(y, bi)) > kResidEps) {
            code = kResidAbs;
          }
          if (code && i < first) { first = i; fcode = code; }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const int of = __shfl_xor_sync(0xffffffffu, first, off);
          const int oc = __shfl_xor_sync(0xffffffffu, fcode, off);
          if (of < first) { first = of; fcode = oc; }
        }
        for (int i = wl; i < n; i += 32) bv.out[ov + i] = xs[i];
        if (wl == 0) {
          bv.status[s] = fcode;
          if (bv.diag) bv.diag[s] = kDiagExact;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace ss
