// CTA-per-system kernels for 32 < n <= 128 (macro-atom jumping matrices of a
// few dozen levels, per-element macro populations).
//
// The padded P x P matrix lives in registers: a TR x TC thread grid where the
// thread (tr, tc) owns rows [tr*RB, tr*RB+RB) and columns [tc*CB, tc*CB+CB);
// a warp covers 32/TC whole thread rows, so every thread finds the owner of
// (its row, column j) in its own warp.  Rows never move; each row carries its
// current position.  Step j:
//   A  owners of column j propose their best (|a_rj|, pos) row, reduced across
//      the owner lanes of each warp by shuffles, one candidate per warp to
//      shared memory;                                          -- barrier
//   B  every thread reduces the per-warp candidates (same answer everywhere),
//      updates row positions, takes its rows' column-j entries from the owner
//      lane by shuffle and forms its own multipliers; the pivot row's owners
//      publish that row;                                      -- barrier
//   C  every thread applies the rank-1 update to its RB x CB block.
// Register indices stay compile-time constants: the element of column j in a
// thread's block is picked with a short predicated chain.
//
// Arithmetic: as in kernels_small.cuh (GSL-exact below-pivot updates; the
// solve's triangular sweeps follow LU_svx's order, run by one warp from a
// shared-memory copy of the factors).
#pragma once
#include "ss_common.cuh"

namespace ss {

// v[c] for a run-time c in [0, W) without dynamic register indexing
template <int W>
__device__ __forceinline__ double pick(const double (&v)[W], int c) {
  double x = v[0];
#pragma unroll
  for (int i = 1; i < W; ++i) x = (c == i) ? v[i] : x;
  return x;
}

template <int KIND, int TR, int TC, int RB, int CB>
struct CtaShape {
  static constexpr int P = TR * RB;
  static constexpr int NT = TR * TC;
  static constexpr int NW = NT / 32;
  static constexpr int LS = P + 1;                          // LU row stride in shared memory
  static constexpr size_t dyn_smem = (KIND == kSolve) ? size_t(P) * LS * sizeof(double) : 0;
  // resident CTAs per SM asked of the register allocator: about 3 registers
  // per owned element plus a fixed ~48 for indices and the step state
  static constexpr int regs = 48 + 3 * RB * CB;
  static constexpr int min_blocks = (65536 / (NT * (regs > 255 ? 255 : regs))) < 1 ? 1 : (65536 / (NT * (regs > 255 ? 255 : regs)));
  static_assert(TC * CB == P, "square padding");
  static_assert(TC <= 32 && (32 % TC) == 0, "column groups tile a warp");
  static_assert(NT % 32 == 0, "whole warps");
};

template <int KIND, int TR, int TC, int RB, int CB>
__global__ void __launch_bounds__(TR * TC, (CtaShape<KIND, TR, TC, RB, CB>::min_blocks))
cta_exact_kernel(BatchView bv) {
  using Sh = CtaShape<KIND, TR, TC, RB, CB>;
  constexpr int P = Sh::P;
  constexpr int NW = Sh::NW;
  constexpr int LS = Sh::LS;

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
  const int grp_lane0 = wl & ~(TC - 1);       // lane of (this thread row, tc = 0)

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

    for (int j = 0; j < n && !sing; ++j) {
      const int jb = j / CB, cj = j - jb * CB;
      // ---- A: candidates of column j --------------------------------------
      double key = -1.0, val = 0.0;
      int pk = 0x7fffffff;                     // (pos << 16) | row
      if (tc == jb) {
#pragma unroll
        for (int r = 0; r < RB; ++r) {
          const int row = row0 + r;
          const double arj = pick<CB>(a[r], cj);
          if (row < n && !((done >> r) & 1u)) {
            const double k = pivot_key(arj);
            const int pp = (pos[r] << 16) | row;
            if (pivot_better(k, pp, key, pk)) { key = k; pk = pp; val = arj; }
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

      // ---- B: the pivot, positions, multipliers, published pivot row -------
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
        sing = true;                           // uniform: every thread read the same ujj
        continue;
      }
      const double rinv = __drcp_rn(ujj);      // correctly rounded, = fl(1/ujj)
      const int prb = p / RB, prr = p - prb * RB;
      // multipliers of this thread's rows; column j lives in lane (tr, jb)
      double lr[RB];
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const double mine = pick<CB>(a[r], cj);
        const double arj = __shfl_sync(0xffffffffu, mine, grp_lane0 + jb);
        const int row = row0 + r;
        double l = 0.0;
        if (row < n && row != p) {
          if (!((was_done >> r) & 1u)) l = gsl_multiplier(arj, ujj, rinv);
          else if (KIND == kInvert) l = mul_rn(arj, rinv);
        }
        lr[r] = l;
      }
      if (tr == prb) {
#pragma unroll
        for (int r = 0; r < RB; ++r)
          if (r == prr) {
#pragma unroll
            for (int c = 0; c < CB; ++c) ubuf[col0 + c] = a[r][c];
          }
      }
      __syncthreads();

      // ---- C: rank-1 update ------------------------------------------------
      double uc[CB];
#pragma unroll
      for (int c = 0; c < CB; ++c) uc[c] = ubuf[col0 + c];
      const bool own_col = (tc == jb);
      if (KIND == kInvert) {
        // rows whose multiplier is 0 (the pivot row, padding) keep their values
#pragma unroll
        for (int r = 0; r < RB; ++r) {
#pragma unroll
          for (int c = 0; c < CB; ++c) a[r][c] = sub_rn(a[r][c], mul_rn(lr[r], uc[c]));
        }
        if (tr == prb) {
#pragma unroll
          for (int r = 0; r < RB; ++r)
            if (r == prr) {
#pragma unroll
              for (int c = 0; c < CB; ++c) a[r][c] = mul_rn(a[r][c], rinv);
            }
        }
        if (own_col) {
          // column j becomes column j of the inverse-in-place: -l, and 1/u_jj on the pivot row
#pragma unroll
          for (int r = 0; r < RB; ++r) {
            const double v = (row0 + r == p) ? rinv : -lr[r];
#pragma unroll
            for (int c = 0; c < CB; ++c)
              if (c == cj) a[r][c] = v;
          }
        }
      } else {
        if (tc >= jb) {
#pragma unroll
          for (int r = 0; r < RB; ++r) {
#pragma unroll
            for (int c = 0; c < CB; ++c)
              if (tc > jb || c > cj) a[r][c] = sub_rn(a[r][c], mul_rn(lr[r], uc[c]));
          }
        }
        if (own_col) {
#pragma unroll
          for (int r = 0; r < RB; ++r) {
            const int row = row0 + r;
            if (row < n && row != p && !((was_done >> r) & 1u)) {
#pragma unroll
              for (int c = 0; c < CB; ++c)
                if (c == cj) a[r][c] = lr[r];
            }
          }
        }
      }
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
        if (bv.diag) bv.diag[s] = kDiagExact;
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
          if (bv.diag) bv.diag[s] = kDiagExact;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace ss
