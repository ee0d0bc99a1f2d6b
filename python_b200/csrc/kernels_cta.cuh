// CTA-per-system kernels for 32 < n <= 128 (macro-atom jumping matrices of a
// few dozen levels, per-element macro populations).
//
// The padded P x P matrix lives in registers: a TR x TC thread grid where the
// thread (tr, tc) owns rows [tr*RB, tr*RB+RB) and columns [tc*CB, tc*CB+CB).
// Rows never move; each row carries its current position.  Step j:
//   A  owners of column j propose their best (|a_rj|, pos) row, reduced across
//      the owner lanes of each warp by shuffles, one candidate per warp to
//      shared memory;                                          -- barrier
//   B  every thread reduces the per-warp candidates (same answer everywhere),
//      updates row positions, the pivot row's owners publish it and the
//      column owners publish the multipliers;                 -- barrier
//   C  every thread applies the rank-1 update to its block.
// The column loop is split into a dynamic block loop and a static CB-wide
// inner loop so every register index is a compile-time constant.
//
// Arithmetic: as in kernels_small.cuh (GSL-exact below-pivot updates; the
// solve's triangular sweeps follow LU_svx's order, run by one warp from a
// shared-memory copy of the factors).
#pragma once
#include "ss_common.cuh"

namespace ss {

template <int KIND, int TR, int TC, int RB, int CB>
struct CtaShape {
  static constexpr int P = TR * RB;
  static constexpr int NT = TR * TC;
  static constexpr int NW = NT / 32;
  static constexpr int LS = P + 1;                          // LU row stride in shared memory
  static constexpr size_t dyn_smem = (KIND == kSolve) ? size_t(P) * LS * sizeof(double) : 0;
  static_assert(TC * CB == P, "square padding");
  static_assert(TC <= 32 && (32 % TC) == 0, "column groups tile a warp");
  static_assert(NT % 32 == 0, "whole warps");
};

template <int KIND, int TR, int TC, int RB, int CB>
__global__ void __launch_bounds__(TR * TC, 1)
cta_exact_kernel(BatchView bv) {
  using Sh = CtaShape<KIND, TR, TC, RB, CB>;
  constexpr int P = Sh::P;
  constexpr int NW = Sh::NW;
  constexpr int LS = Sh::LS;

  __shared__ __align__(16) double lbuf[P];
  __shared__ __align__(16) double ubuf[P];
  __shared__ double ckey[NW], cval[NW];
  __shared__ int cpk[NW];
  __shared__ int ipiv[P];
  __shared__ int cmap[P];
  __shared__ int csrc[P];
  __shared__ double vec[P];
  __shared__ double xs[P];
  extern __shared__ __align__(16) double lu_s[];

  const int t = threadIdx.x;
  const int tr = t / TC, tc = t % TC;
  const int wid = t >> 5, wl = t & 31;
  const int row0 = tr * RB, col0 = tc * CB;

  for (int item = blockIdx.x; item < bv.count; item += gridDim.x) {
    const int s = bv.list[item];
    const int n = bv.n[s];
    const double* __restrict__ Ag = bv.A + bv.offA[s];

    double a[RB][CB];
    int pos[RB];
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int row = row0 + r;
      pos[r] = row;
#pragma unroll
      for (int c = 0; c < CB; ++c) {
        const int col = col0 + c;
        a[r][c] = (row < n && col < n) ? Ag[int64_t(row) * n + col] : 0.0;
      }
    }
    unsigned done = 0;
    bool sing = false;
    const int nblk = (n + CB - 1) / CB;

    for (int jb = 0; jb < nblk && !sing; ++jb) {
#pragma unroll
      for (int cj = 0; cj < CB; ++cj) {
        const int j = jb * CB + cj;
        if (j < n && !sing) {
          // ---- A: candidates of column j --------------------------------
          double key = -1.0, val = 0.0;
          int pk = 0x7fffffff;                     // (pos << 16) | row
          if (tc == jb) {
#pragma unroll
            for (int r = 0; r < RB; ++r) {
              const int row = row0 + r;
              if (row < n && !((done >> r) & 1u)) {
                const double k = pivot_key(a[r][cj]);
                const int pp = (pos[r] << 16) | row;
                if (pivot_better(k, pp, key, pk)) { key = k; pk = pp; val = a[r][cj]; }
              }
            }
          }
#pragma unroll
          for (int off = TC; off < 32; off <<= 1) {
            const double ok = __shfl_xor_sync(0xffffffffu, key, off);
            const double ov = __shfl_xor_sync(0xffffffffu, val, off);
            const int op = __shfl_xor_sync(0xffffffffu, pk, off);
            if (pivot_better(ok, op, key, pk)) { key = ok; pk = op; val = ov; }
          }
          if (wl == jb) { ckey[wid] = key; cval[wid] = val; cpk[wid] = pk; }
          __syncthreads();

          // ---- B: the pivot, positions, published row and multipliers ---
          key = -1.0; pk = 0x7fffffff; val = 0.0;
#pragma unroll
          for (int w = 0; w < NW; ++w) {
            const double k = ckey[w];
            const int pp = cpk[w];
            if (pivot_better(k, pp, key, pk)) { key = k; pk = pp; val = cval[w]; }
          }
          const int p = pk & 0xffff, ppos = pk >> 16;
          const double ujj = val;
          const unsigned was_done = done;
#pragma unroll
          for (int r = 0; r < RB; ++r) {
            if (row0 + r == p) { pos[r] = j; done |= 1u << r; }
            else if (pos[r] == j) pos[r] = ppos;
          }
          if (t == 0) ipiv[j] = ppos;
          if (ujj == 0.0) {
            sing = true;
          } else {
            const double rinv = div_rn(1.0, ujj);
            const int prb = p / RB, prr = p - prb * RB;
            if (tr == prb) {
#pragma unroll
              for (int r = 0; r < RB; ++r)
                if (r == prr) {
#pragma unroll
                  for (int c = 0; c < CB; ++c) ubuf[col0 + c] = a[r][c];
                }
            }
            if (tc == jb) {
#pragma unroll
              for (int r = 0; r < RB; ++r) {
                const int row = row0 + r;
                double l = 0.0;
                if (row < n && row != p) {
                  if (!((was_done >> r) & 1u)) l = gsl_multiplier(a[r][cj], ujj, rinv);
                  else if (KIND == kInvert) l = mul_rn(a[r][cj], rinv);
                }
                lbuf[row] = l;
              }
            }
            __syncthreads();

            // ---- C: rank-1 update ----------------------------------------
            double lr[RB], uc[CB];
#pragma unroll
            for (int r = 0; r < RB; ++r) lr[r] = lbuf[row0 + r];
#pragma unroll
            for (int c = 0; c < CB; ++c) uc[c] = ubuf[col0 + c];
            if (KIND == kInvert) {
#pragma unroll
              for (int r = 0; r < RB; ++r) {
                if (lr[r] != 0.0) {
#pragma unroll
                  for (int c = 0; c < CB; ++c)
                    if (!(tc == jb && c == cj)) a[r][c] = sub_rn(a[r][c], mul_rn(lr[r], uc[c]));
                }
              }
              if (tr == prb) {
#pragma unroll
                for (int r = 0; r < RB; ++r)
                  if (r == prr) {
#pragma unroll
                    for (int c = 0; c < CB; ++c) a[r][c] = mul_rn(a[r][c], rinv);
                  }
              }
              if (tc == jb) {
#pragma unroll
                for (int r = 0; r < RB; ++r) {
                  const int row = row0 + r;
                  if (row < n) a[r][cj] = (row == p) ? rinv : -lr[r];
                }
              }
            } else {
              if (tc >= jb) {
#pragma unroll
                for (int r = 0; r < RB; ++r) {
                  if (lr[r] != 0.0) {
#pragma unroll
                    for (int c = 0; c < CB; ++c)
                      if (tc > jb || c > cj) a[r][c] = sub_rn(a[r][c], mul_rn(lr[r], uc[c]));
                  }
                }
              }
              if (tc == jb) {
#pragma unroll
                for (int r = 0; r < RB; ++r) {
                  const int row = row0 + r;
                  if (row < n && row != p && !((was_done >> r) & 1u)) a[r][cj] = lr[r];
                }
              }
            }
          }
        }
      }
    }

    if (sing) {
      if (t == 0) {
        bv.status[s] = (KIND == kSolve) ? kSolveSingular : kInvertSingular;
        if (bv.diag) bv.diag[s] = 0;
      }
      __syncthreads();
      continue;
    }

    if (KIND == kInvert) {
      // reverse-order column unscramble: output column cmap[k] takes column k
      if (t == 0) {
        for (int c = 0; c < n; ++c) csrc[c] = c;
        for (int jj = n - 1; jj >= 0; --jj) {
          const int q = ipiv[jj];
          if (q != jj) { const int tmp = csrc[jj]; csrc[jj] = csrc[q]; csrc[q] = tmp; }
        }
        for (int c = 0; c < n; ++c) cmap[csrc[c]] = c;
      }
      __syncthreads();
      double* __restrict__ Og = bv.out + bv.offA[s];
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int row = row0 + r;
        if (row < n) {
          const int64_t ro = int64_t(pos[r]) * n;
#pragma unroll
          for (int c = 0; c < CB; ++c) {
            const int col = col0 + c;
            if (col < n) Og[ro + cmap[col]] = a[r][c];
          }
        }
      }
      if (t == 0) {
        bv.status[s] = kOk;
        if (bv.diag) bv.diag[s] = 0;
      }
    } else {
      // factors into shared memory by position; cmap[i] = original row at position i
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int row = row0 + r;
        if (row < n) {
#pragma unroll
          for (int c = 0; c < CB; ++c) lu_s[pos[r] * LS + col0 + c] = a[r][c];
          if (tc == 0) cmap[pos[r]] = row;
        }
      }
      __syncthreads();
      if (wid == 0) {
        const int64_t ov = bv.offv[s];
        for (int i = wl; i < n; i += 32) vec[i] = bv.b[ov + cmap[i]];
        __syncwarp();
        // forward sweep (unit L), ascending j per entry
        for (int j = 0; j < n; ++j) {
          const double yj = vec[j];
          for (int i = j + 1 + wl; i < n; i += 32) vec[i] = sub_rn(vec[i], mul_rn(lu_s[i * LS + j], yj));
          __syncwarp();
        }
        // backward sweep in LU_svx's order (serial chain)
        if (wl == 0) {
          for (int i = n - 1; i >= 0; --i) {
            double u = vec[i];
            for (int k = i + 1; k < n; ++k) u = sub_rn(u, mul_rn(lu_s[i * LS + k], xs[k]));
            xs[i] = div_rn(u, lu_s[i * LS + i]);
          }
        }
        __syncwarp();
        // residual check on the original A, first failing row decides
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
          if (bv.diag) bv.diag[s] = 0;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace ss
