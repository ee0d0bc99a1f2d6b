// Certified inverse for orders above the register-resident classes (217 ..
// 1024): blocked Gauss-Jordan without pivoting, streamed through global
// memory, its updates on the FP64 tensor-core MMA.
//
// The certificate and the reason no pivoting is needed are those of
// kernels_cert.cuh (nonsingular M-matrices with a relative row-dominance margin
// of kCertMargin; the macro-atom matrices of calc_matom_matrix,
// source/macro_accelerate.c:268-284, inverted at :315).  A matrix that fails
// it is appended to the fallback list of its GSL-exact class.
//
// One CTA inverts one matrix at a time, in place in the output: the matrices
// are taken from a queue, largest first (an atomic counter over the bucket's
// list, which the host sorts by order).  Steps of BT = 64 pivot columns, K =
// [k0, k0 + kb):
//   D    the pivot block W[K][K] is inverted by the CTA (unpivoted Gauss-Jordan
//        on 64 x 64, a column of 32 entries per thread, one barrier per pivot);
//   R'   the pivot rows become D^-1 W[K][:] (on K's own tile: D^-1 I), tile by
//        tile;
//   W    every other 64-row tile I: W[I][:] <- W[I][:] - W[I][K] R', where the
//        old W[I][K] is held negated in shared memory before the pass and the
//        tile of K's columns starts from zero, so that it becomes -W[I][K] D^-1.
// A 64 x 64 tile update is 4 x 4 sub-blocks of 8 x 8 per warp (a 2 x 2 warp
// grid), each the accumulator fragment of mma.sync m8n8k4 f64, with both
// operand tiles in shared memory (row stride 68 doubles: the fragment loads of
// a half-warp fall on distinct banks).  Every W element is read and written
// once per step, so the traffic is 16 n^2 bytes per step against 2 n^2 BT
// flops: 8 flops per byte, above the B200's FP64-to-HBM balance of ~5.5.  Each
// CTA holds two tiles (70 KB of shared memory) and three run per SM, whose
// loads, barriers and pivot-block inverses overlap one another's MMAs.
// With the macro-atom epilogue (CertEpi) the last step writes B = N^-1 diag(R)
// (the pivot rows after the step, since their unscaled values feed it), and
// the row running totals follow in 32 x 32 tiles.
#pragma once
#include "kernels_cert.cuh"

namespace ss {

template <int MINB_>
struct CgjlShape {
  static constexpr int BT = 64;        // pivot columns per step; tile edge
  static constexpr int NTH = 128;      // 4 warps, a 2 x 2 grid of 32 x 32 sub-tiles
  static constexpr int SA = 68;        // shared tile row stride (doubles)
  static constexpr int MINB = MINB_;   // CTAs per SM asked of the register allocator
  static constexpr int off_A = 0;                 // [BT][SA] A operand: D^-1, or -W[I][K]
  static constexpr int off_B = BT * SA;           // [BT][SA] B operand: W[K][J], or R'[K][J]
  static constexpr int off_x = 2 * BT * SA;       // [2][BT] pivot row, [2][BT] pivot column
  static constexpr int off_slot = off_x + 4 * BT; // queue item broadcast
  static constexpr int n_dbl = off_slot + 2;
  static constexpr size_t dyn_smem = size_t(n_dbl) * 8;
  static_assert(4 * (32 * 33) <= 2 * BT * SA, "running-total tiles fit the operand buffers");
};

namespace cgjl {

constexpr int BT = 64, SA = 68;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// tile [r0, r0 + rb) x [c0, c0 + cb) of an n x n row-major matrix into a BT x BT
// shared tile, zero outside (identity on the diagonal when ident), negated
// when neg
__device__ __forceinline__ void load_tile(double* __restrict__ dst, const double* src, int n, int r0, int rb,
                                          int c0, int cb, bool ident, bool neg, int tid) {
  double v[32];
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    const int e = tid + 128 * m, r = e >> 6, c = e & 63;
    v[m] = (r < rb && c < cb) ? src[int64_t(r0 + r) * n + c0 + c] : 0.0;
  }
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    const int e = tid + 128 * m, r = e >> 6, c = e & 63;
    double x = neg ? -v[m] : v[m];
    if (ident) x = (r == c && r < rb) ? 1.0 : 0.0;
    dst[r * SA + c] = x;
  }
}

// acc += A B over the 64-deep tiles: warp (wr, wc) covers rows 32 wr .. +32,
// columns 32 wc .. +32 in 4 x 4 fragments
__device__ __forceinline__ void mma_tile(double (&acc)[4][4][2], const double* __restrict__ As,
                                         const double* __restrict__ Bs, int wr, int wc, int g, int t) {
#pragma unroll 4
  for (int kk = 0; kk < BT / 4; ++kk) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = As[(32 * wr + 8 * i + g) * SA + 4 * kk + t];
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = Bs[(4 * kk + t) * SA + 32 * wc + 8 * j + g];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma_884(acc[i][j], a[i], b[j]);
  }
}

}  // namespace cgjl

template <int MINB>
__global__ void __launch_bounds__(128, MINB)
    cgjl_inverse_kernel(BatchView bv, CertArgs ca, CertEpi ep, int* __restrict__ queue) {
  using namespace cgjl;
  using S = CgjlShape<MINB>;
  extern __shared__ __align__(16) double sm[];
  double* As = sm + S::off_A;
  double* Bs = sm + S::off_B;
  double* xr = sm + S::off_x;       // pivot rows, by parity of the pivot
  double* xc = xr + 2 * BT;         // pivot columns, by parity
  int* slot = reinterpret_cast<int*>(sm + S::off_slot);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = warp >> 1, wc = warp & 1;
  const int cnt = batch_count(bv);

  for (;;) {
    if (tid == 0) *slot = atomicAdd(queue, 1);
    __syncthreads();
    const int item = *slot;
    __syncthreads();
    if (item >= cnt) break;
    const int s = bv.list[item];
    const int n = bv.n[s];
    const double* Ag = bv.A + bv.offA[s];
    double* Wg = bv.out + bv.offA[s];

    // ---- certificate, a warp per row (coalesced)
    bool ok = true;
    for (int r = warp; r < n; r += 4) {
      const double* row = Ag + int64_t(r) * n;
      double off = 0.0;
      for (int c = lane; c < n; c += 32) {
        const double a = row[c];
        if (c != r) {
          ok &= (a <= 0.0);   // false for NaN
          off += fabs(a);
        }
      }
      off = warp_sum(off);
      const double d = row[r];
      ok &= (d > 0.0) && (d < INFINITY) && (off * (1.0 + 0x1p-40) <= (1.0 - kCertMargin) * d);
    }
    if (!__syncthreads_and(int(ok))) {
      if (tid == 0) {
        const int cls = ca.xcls[s];
        const int k = atomicAdd(ca.fb_count + cls, 1);
        ca.fb_list[ca.fb_off[cls] + k] = s;
      }
      continue;
    }

    const int nb = (n + BT - 1) / BT;
    for (int kt = 0; kt < nb; ++kt) {
      const int k0 = kt * BT, kb = min(BT, n - k0);
      const double* src = (kt == 0) ? Ag : Wg;   // the first step reads the input

      // ---- D^-1: thread (column c, rows 32 h ..) of the padded 64 x 64 block
      {
        const int c = tid & 63, h = tid >> 6;
        double dv[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int r = 32 * h + i;
          dv[i] = (r < kb && c < kb) ? src[int64_t(k0 + r) * n + k0 + c] : (r == c ? 1.0 : 0.0);
        }
#pragma unroll
        for (int j = 0; j < BT; ++j) {
          double* rx = xr + (j & 1) * BT;
          double* cx = xc + (j & 1) * BT;
          if (h == (j >> 5)) rx[c] = dv[j & 31];
          if (c == j) {
#pragma unroll
            for (int i = 0; i < 32; ++i) cx[32 * h + i] = dv[i];
          }
          __syncthreads();
          const double p = 1.0 / rx[j];
          const double rj = rx[c] * p;
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const int r = 32 * h + i;
            if (r == j) {
              dv[i] = (c == j) ? p : rj;
            } else {
              const double f = cx[r];
              dv[i] = (c == j) ? -f * p : fma(-f, rj, dv[i]);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) As[(32 * h + i) * SA + c] = dv[i];
      }

      // ---- R' = D^-1 W[K][J] on the pivot rows (D^-1 on K's own tile)
      for (int jt = 0; jt < nb; ++jt) {
        const int j0 = jt * BT, jb = min(BT, n - j0);
        load_tile(Bs, src, n, k0, kb, j0, jb, jt == kt, false, tid);
        __syncthreads();
        double acc[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
        mma_tile(acc, As, Bs, wr, wc, g, t);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = 32 * wr + 8 * i + g;
          if (r < kb) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int c = 32 * wc + 8 * j + 2 * t + e;
                if (c < jb) Wg[int64_t(k0 + r) * n + j0 + c] = acc[i][j][e];
              }
          }
        }
        __syncthreads();
      }

      // ---- every other row tile: W[I][:] += (-W[I][K]) R'
      const bool last = (kt == nb - 1);
      const double* __restrict__ Rs = (last && ep.R) ? ep.R + ep.offv[s] : nullptr;
      for (int it = 0; it < nb; ++it) {
        if (it == kt) continue;
        const int i0 = it * BT, ib = min(BT, n - i0);
        load_tile(As, src, n, i0, ib, k0, kb, false, true, tid);
        for (int jt = 0; jt < nb; ++jt) {
          const int j0 = jt * BT, jb = min(BT, n - j0);
          // the tile's own values first (HBM), then R' (L2): both in flight at once
          double acc[4][4][2];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int r = 32 * wr + 8 * i + g;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int c = 32 * wc + 8 * j + 2 * t + e;
                acc[i][j][e] = (jt != kt && r < ib && c < jb) ? src[int64_t(i0 + r) * n + j0 + c] : 0.0;
              }
          }
          load_tile(Bs, Wg, n, k0, kb, j0, jb, false, false, tid);
          __syncthreads();
          mma_tile(acc, As, Bs, wr, wc, g, t);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int r = 32 * wr + 8 * i + g;
            if (r < ib) {
#pragma unroll
              for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                  const int c = 32 * wc + 8 * j + 2 * t + e;
                  if (c < jb) {
                    const double w = acc[i][j][e];
                    Wg[int64_t(i0 + r) * n + j0 + c] = Rs ? mul_rn(w, __ldg(Rs + j0 + c)) : w;
                  }
                }
            }
          }
          __syncthreads();
        }
      }
      // the pivot rows of the last step, scaled now that no tile reads them
      if (Rs) {
        for (int e = tid; e < kb * n; e += S::NTH) {
          const int r = e / n, c = e - r * n;
          double* w = Wg + int64_t(k0 + r) * n + c;
          *w = mul_rn(*w, __ldg(Rs + c));
        }
        __syncthreads();
      }
    }

    // ---- row running totals of B (32 x 32 tiles through shared memory, each
    // lane adding its own row left to right)
    if (ep.C) {
      double* __restrict__ Cg = ep.C + bv.offA[s];
      double* tl = sm + warp * (32 * 33);
      for (int r0 = 32 * warp; r0 < n; r0 += 128) {
        double total = 0.0;
        for (int c0 = 0; c0 < n; c0 += 32) {
          const int c = c0 + lane;
#pragma unroll 8
          for (int k = 0; k < 32; ++k) {
            const int rk = r0 + k;
            tl[k * 33 + lane] = (rk < n && c < n) ? __ldcg(Wg + int64_t(rk) * n + c) : 0.0;
          }
          __syncwarp();
          const int cm = min(32, n - c0);
          for (int k = 0; k < cm; ++k) {
            total = add_rn(total, tl[lane * 33 + k]);
            tl[lane * 33 + k] = total;
          }
          __syncwarp();
#pragma unroll 8
          for (int k = 0; k < 32; ++k) {
            const int rk = r0 + k;
            if (rk < n && c < n) Cg[int64_t(rk) * n + c] = tl[k * 33 + lane];
          }
          __syncwarp();
        }
      }
      __syncthreads();
    }
    if (tid == 0) {
      bv.status[s] = kOk;
      if (bv.diag) bv.diag[s] = 0;
    }
  }
}

}  // namespace ss
