// CTA-per-system kernels for n > 256 (large macro atoms, full ion matrices).
//
// The system is factorised in a global-memory workspace W (the output buffer
// for an inverse, a per-CTA scratch slab for a solve; a few hundred systems
// are in flight, so W stays in L2), panel by panel of NB columns:
//   1. the n x NB panel is staged in shared memory and factorised there by all
//      warps with physical row swaps (first strict maximum, as GSL's idamax),
//      recording the multipliers M (n x NB) of every row at every panel step;
//   2. for every other column: the panel's row swaps (lu.c:263 apply_pivots),
//      then the pivot rows' values at their own step by the unit-lower
//      recurrence V_k = W_k - sum_{k'<k} M[k][k'] V_k' (the dtrsm of lu.c:266);
//   3. W -= M V over the rest of the matrix in 4 x 4 register tiles, k ascending
//      (the dgemm of lu.c:269), one rounding per product and per difference in
//      the LU region (rows below the panel, columns right of it).
// Each entry of the LU region therefore sees exactly GSL's sequence of
// operations.  For an inverse the same sweep also eliminates the rows above
// the pivots and the already-inverted columns (blocked Gauss-Jordan; fused
// multiply-add there), the pivot rows are scaled by 1/u_kk, and the columns are
// permuted at the end (A^-1 = W P).
#pragma once
#include "ss_common.cuh"

namespace ss {

constexpr int kGThreads = 256;
constexpr int kGTile = 4;                               // register tile edge of the update
constexpr int kGTileRows = 16 * kGTile;                 // 16 x 16 threads -> 64 x 64 elements per pass

// panel width for a bucket whose largest order is nmax
__host__ __device__ constexpr int global_panel_width(int nmax) { return nmax <= 512 ? 16 : 8; }

__host__ __device__ constexpr size_t global_smem_bytes_nb(int nmax, int nb) {
  return size_t(2) * nmax * (nb + 1) * sizeof(double)  // panel + multipliers
       + size_t(nb) * nmax * sizeof(double)            // V for every column
       + size_t(nb + 16) * sizeof(double)              // 1/u_kk, warp candidates
       + size_t(2) * nmax * sizeof(int) + 64;          // pivots, permutation, warp rows
}
__host__ __device__ constexpr size_t global_smem_bytes(int nmax) {
  return global_smem_bytes_nb(nmax, global_panel_width(nmax));
}

// DIRECT = true is the variant behind solve_matrix_batched_noalloc: system
// `item` is batch entry `item` (no bucket list) and a system larger than nmax
// is refused with status -1 instead of being factorised.
template <int KIND, int NB, bool DIRECT = false>
__global__ void __launch_bounds__(kGThreads, 1)
global_exact_kernel(BatchView bv, int nmax, double* scratch, int64_t slab) {
  constexpr int PS = NB + 1;
  extern __shared__ __align__(16) double gsm[];
  double* Ps = gsm;                                   // [nmax][PS] panel
  double* Ms = Ps + size_t(nmax) * PS;                // [nmax][PS] multipliers
  double* Vs = Ms + size_t(nmax) * PS;                // [NB][nmax] pivot rows at their step
  double* rinv_s = Vs + size_t(NB) * nmax;            // [NB]
  double* red_k = rinv_s + NB;                        // [8] warp candidates
  int* ipiv = reinterpret_cast<int*>(red_k + 16);     // [nmax]
  int* perm = ipiv + nmax;                            // [nmax]
  __shared__ int mv_src[2 * NB], mv_dst[2 * NB], mv_cnt[1];
  __shared__ int red_r[kGThreads / 32];

  const int t = threadIdx.x;
  const int wid = t >> 5, wl = t & 31;
  const int tr = t >> 4, tc = t & 15;                 // 16 x 16 thread grid of the update

  const int count = batch_count(bv);
  for (int item = blockIdx.x; item < count; item += gridDim.x) {
    const int s = DIRECT ? item : bv.list[item];
    const int n = bv.n[s];
    if (DIRECT && (n < 1 || n > nmax)) {
      if (t == 0) bv.status[s] = -1;
      continue;
    }
    const double* __restrict__ Ag = bv.A + bv.offA[s];
    double* __restrict__ W = (KIND == kInvert) ? bv.out + bv.offA[s] : scratch + int64_t(blockIdx.x) * slab;
    const int64_t nn = int64_t(n) * n;
    for (int64_t e0 = t; e0 < nn; e0 += 8 * kGThreads) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = (e0 + u * kGThreads < nn) ? __ldg(Ag + e0 + u * kGThreads) : 0.0;
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (e0 + u * kGThreads < nn) W[e0 + u * kGThreads] = v[u];
    }
    __syncthreads();

    // every thread reads the same pivot after a barrier, so `sing` is uniform
    bool sing = false;
    for (int j0 = 0; j0 < n; j0 += NB) {
      const int nb = min(NB, n - j0);
      // ---- 1. the panel, factorised in shared memory by all warps ----------
      for (int e0 = t; e0 < n * NB; e0 += 8 * kGThreads) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int e = e0 + u * kGThreads, r = e / NB, k = e - r * NB;
          v[u] = (e < n * NB && k < nb) ? W[int64_t(r) * n + j0 + k] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int e = e0 + u * kGThreads, r = e / NB, k = e - r * NB;
          if (e < n * NB) { Ps[r * PS + k] = v[u]; Ms[r * PS + k] = 0.0; }
        }
      }
      if (t < NB) rinv_s[t] = 0.0;
      __syncthreads();
      for (int k = 0; k < nb; ++k) {
        const int j = j0 + k;
        double bk = -1.0;
        int br = 0x7fffffff;
        for (int r = j + t; r < n; r += kGThreads) {
          const double key = pivot_key(Ps[r * PS + k]);
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
          if (t < NB) {
            const double x = Ps[j * PS + t]; Ps[j * PS + t] = Ps[p * PS + t]; Ps[p * PS + t] = x;
          } else if (t < 2 * NB) {
            const int c = t - NB;
            const double x = Ms[j * PS + c]; Ms[j * PS + c] = Ms[p * PS + c]; Ms[p * PS + c] = x;
          }
        }
        __syncthreads();
        const double ujj = Ps[j * PS + k];
        if (ujj == 0.0) {
          sing = true;
          break;
        }
        const double rinv = __drcp_rn(ujj);   // correctly rounded, = fl(1/ujj)
        double piv[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) piv[c] = Ps[j * PS + c];
        __syncthreads();
        for (int r = t; r < n; r += kGThreads) {
          if (r == j || (KIND == kSolve && r < j)) continue;
          double row[NB];
#pragma unroll
          for (int c = 0; c < NB; ++c) row[c] = Ps[r * PS + c];
          const double v = Ps[r * PS + k];
          const bool below = r > j;
          const double l = below ? gsl_multiplier(v, ujj, rinv) : mul_rn(v, rinv);
#pragma unroll
          for (int c = 0; c < NB; ++c) {
            const bool skip = (c == k) || (KIND == kSolve && c < k);
            const double upd = (below && c > k) ? sub_rn(row[c], mul_rn(l, piv[c])) : fma(-l, piv[c], row[c]);
            row[c] = (c == k) ? ((KIND == kInvert) ? -l : l) : (skip ? row[c] : upd);
          }
          Ms[r * PS + k] = l;
#pragma unroll
          for (int c = 0; c < NB; ++c) Ps[r * PS + c] = row[c];
        }
        if (t == 0) {
          rinv_s[k] = rinv;
          if (KIND == kInvert) {
#pragma unroll
            for (int c = 0; c < NB; ++c) Ps[j * PS + c] = (c == k) ? rinv : mul_rn(piv[c], rinv);
          }
        }
        __syncthreads();
      }
      if (sing) break;
      for (int e = t; e < n * NB; e += kGThreads) {
        const int r = e / NB, k = e - r * NB;
        if (k < nb) W[int64_t(r) * n + j0 + k] = Ps[r * PS + k];
      }

      // ---- 2. swaps and V for every other column -----------------------------
      // the panel's swaps as one gather: row mv_dst[m] takes the old row mv_src[m]
      if (t == 0) {
        int m = 0;
        for (int k = 0; k < nb; ++k) perm[j0 + k] = j0 + k;
        for (int k = 0; k < nb; ++k) {
          const int q = ipiv[j0 + k];
          if (q >= j0 + nb) perm[q] = q;   // rows below the panel that take part
        }
        for (int k = 0; k < nb; ++k) {
          const int q = ipiv[j0 + k];
          if (q != j0 + k) { const int x = perm[j0 + k]; perm[j0 + k] = perm[q]; perm[q] = x; }
        }
        for (int k = 0; k < nb; ++k) {
          const int rr = j0 + k;
          if (perm[rr] != rr) { mv_dst[m] = rr; mv_src[m] = perm[rr]; ++m; }
          const int q = ipiv[rr];
          if (q >= j0 + nb && perm[q] != q) {
            bool seen = false;
            for (int x = 0; x < m; ++x) seen = seen || (mv_dst[x] == q);
            if (!seen) { mv_dst[m] = q; mv_src[m] = perm[q]; ++m; }
          }
        }
        mv_cnt[0] = m;
      }
      __syncthreads();
      const int nmv = mv_cnt[0];
      // (a solve leaves the L part of earlier panels alone apart from the swaps)
      for (int c = t; c < n; c += kGThreads) {
        if (c >= j0 && c < j0 + nb) continue;
        double mvv[2 * NB];
#pragma unroll
        for (int m = 0; m < 2 * NB; ++m) mvv[m] = (m < nmv) ? W[int64_t(mv_src[m]) * n + c] : 0.0;
#pragma unroll
        for (int m = 0; m < 2 * NB; ++m)
          if (m < nmv) W[int64_t(mv_dst[m]) * n + c] = mvv[m];
        if (KIND == kInvert || c >= j0 + nb) {
          double vk[NB];
#pragma unroll
          for (int k = 0; k < NB; ++k) vk[k] = (k < nb) ? W[int64_t(j0 + k) * n + c] : 0.0;
#pragma unroll
          for (int k = 1; k < NB; ++k) {
            double v = vk[k];
#pragma unroll
            for (int kk = 0; kk < k; ++kk) v = sub_rn(v, mul_rn(Ms[(j0 + k) * PS + kk], vk[kk]));
            vk[k] = v;
          }
#pragma unroll
          for (int k = 0; k < NB; ++k) Vs[k * nmax + c] = vk[k];
        }
      }
      __syncthreads();

      // ---- 3. W -= M V over the rest, 4 x 4 register tiles -------------------
      // thread (tr, tc) of a 64 x 64 tile owns rows tr*4 .. tr*4+3 and columns
      // tc, tc+16, tc+32, tc+48: V reads are conflict-free, W accesses coalesced
      const int c_lo = (KIND == kInvert) ? 0 : j0 + nb;
      const int r_lo = (KIND == kInvert) ? 0 : j0;
      const int ntc = (n - c_lo + kGTileRows - 1) / kGTileRows;
      const int ntr = (n - r_lo + kGTileRows - 1) / kGTileRows;
      for (int tt = 0; tt < ntc * ntr; ++tt) {
        const int rb = r_lo + (tt / ntc) * kGTileRows + tr * kGTile;
        const int cb = c_lo + (tt % ntc) * kGTileRows + tc;
        int cols[kGTile], ccl[kGTile];
        bool cok[kGTile], cright[kGTile];
        bool all_right = true;
#pragma unroll
        for (int c = 0; c < kGTile; ++c) {
          cols[c] = cb + 16 * c;
          ccl[c] = min(cols[c], n - 1);              // in-range read for lanes whose column is not stored
          cok[c] = cols[c] < n && !(cols[c] >= j0 && cols[c] < j0 + nb);
          cright[c] = cok[c] && cols[c] >= j0 + nb;
          all_right = all_right && (cright[c] || !cok[c]);
        }
        bool rok[kGTile], rpiv[kGTile], rbelow[kGTile];
        bool all_below = true, none_piv = true, none_below = true;
#pragma unroll
        for (int rr = 0; rr < kGTile; ++rr) {
          const int r = rb + rr;
          rok[rr] = r < n;
          rpiv[rr] = rok[rr] && r >= j0 && r < j0 + nb;
          rbelow[rr] = rok[rr] && r >= j0 + nb;
          all_below = all_below && (rbelow[rr] || !rok[rr]);
          none_piv = none_piv && !rpiv[rr];
          none_below = none_below && !rbelow[rr];
        }
        // all 16 loads of the tile first, then the arithmetic, then the stores
        double w[kGTile][kGTile];
#pragma unroll
        for (int rr = 0; rr < kGTile; ++rr) {
          const int rcl = min(rb + rr, n - 1);
#pragma unroll
          for (int c = 0; c < kGTile; ++c) w[rr][c] = W[int64_t(rcl) * n + ccl[c]];
        }
        if (all_below && all_right) {
          // GSL's LU region: one rounding per product and per difference, k ascending
#pragma unroll
          for (int k = 0; k < NB; ++k) {
            double vk[kGTile], mk[kGTile];
#pragma unroll
            for (int c = 0; c < kGTile; ++c) vk[c] = Vs[k * nmax + ccl[c]];
#pragma unroll
            for (int rr = 0; rr < kGTile; ++rr) mk[rr] = Ms[min(rb + rr, n - 1) * PS + k];
#pragma unroll
            for (int rr = 0; rr < kGTile; ++rr)
#pragma unroll
              for (int c = 0; c < kGTile; ++c) w[rr][c] = sub_rn(w[rr][c], mul_rn(mk[rr], vk[c]));
          }
        } else if (KIND == kInvert && none_below && none_piv) {
          // rows above the panel: outside the LU region
#pragma unroll
          for (int k = 0; k < NB; ++k) {
            double vk[kGTile], mk[kGTile];
#pragma unroll
            for (int c = 0; c < kGTile; ++c) vk[c] = Vs[k * nmax + ccl[c]];
#pragma unroll
            for (int rr = 0; rr < kGTile; ++rr) mk[rr] = Ms[min(rb + rr, n - 1) * PS + k];
#pragma unroll
            for (int rr = 0; rr < kGTile; ++rr)
#pragma unroll
              for (int c = 0; c < kGTile; ++c) w[rr][c] = fma(-mk[rr], vk[c], w[rr][c]);
          }
        } else {
          // mixed tile: per element, pivot rows left for the formula below
#pragma unroll
          for (int k = 0; k < NB; ++k) {
            double vk[kGTile], mk[kGTile];
#pragma unroll
            for (int c = 0; c < kGTile; ++c) vk[c] = Vs[k * nmax + ccl[c]];
#pragma unroll
            for (int rr = 0; rr < kGTile; ++rr) mk[rr] = Ms[min(rb + rr, n - 1) * PS + k];
#pragma unroll
            for (int rr = 0; rr < kGTile; ++rr)
#pragma unroll
              for (int c = 0; c < kGTile; ++c) {
                if (rpiv[rr]) continue;
                if (rbelow[rr] && cright[c]) w[rr][c] = sub_rn(w[rr][c], mul_rn(mk[rr], vk[c]));
                else if (KIND == kInvert) w[rr][c] = fma(-mk[rr], vk[c], w[rr][c]);
              }
          }
          // the panel's pivot rows: their value at their own step, then (inverse)
          // scaled and eliminated by the later pivots of the panel
#pragma unroll
          for (int rr = 0; rr < kGTile; ++rr) {
            if (!rpiv[rr]) continue;
            const int r = rb + rr, k = r - j0;
#pragma unroll
            for (int c = 0; c < kGTile; ++c) {
              double acc = Vs[k * nmax + ccl[c]];
              if (KIND == kInvert) {
                acc = acc * rinv_s[k];
                for (int k2 = k + 1; k2 < nb; ++k2) acc = fma(-Ms[r * PS + k2], Vs[k2 * nmax + ccl[c]], acc);
              }
              w[rr][c] = acc;
            }
          }
        }
#pragma unroll
        for (int rr = 0; rr < kGTile; ++rr) {
          if (!rok[rr]) continue;
          const int r = rb + rr;
#pragma unroll
          for (int c = 0; c < kGTile; ++c)
            if (cok[c] && (KIND == kInvert || rbelow[rr] || rpiv[rr])) W[int64_t(r) * n + cols[c]] = w[rr][c];
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

    // GSL's permutation (lu.c:95-109): perm[i] = original row now at row i
    if (t == 0) {
      for (int i = 0; i < n; ++i) perm[i] = i;
      for (int i = 0; i < n; ++i) {
        const int q = ipiv[i];
        if (perm[q] != perm[i]) { const int x = perm[q]; perm[q] = perm[i]; perm[i] = x; }
      }
    }
    __syncthreads();

    if (KIND == kInvert) {
      // A^-1 = W P: column perm[i] of the result is column i of W, row by row
      double* rowbuf = Ps + size_t(wid) * nmax;       // 8 warps x n doubles fit in the panel area
      for (int r = wid; r < n; r += kGThreads / 32) {
        double* w = W + int64_t(r) * n;
        for (int c = wl; c < n; c += 32) rowbuf[perm[c]] = w[c];
        __syncwarp();
        for (int c = wl; c < n; c += 32) w[c] = rowbuf[c];
        __syncwarp();
      }
      if (t == 0) {
        bv.status[s] = kOk;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
    } else {
      double* vec = Ps;                 // y, then x (natural order), n doubles each
      double* xs = Ps + nmax;
      if (wid == 0) {
        const int64_t ov = bv.offv[s];
        for (int i = wl; i < n; i += 32) vec[i] = bv.b[ov + perm[i]];
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
