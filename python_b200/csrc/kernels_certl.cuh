// Certified inverse for orders above the register-resident classes (225 ..
// 1024): blocked Gauss-Jordan without pivoting, streamed through global
// memory, its updates on the FP64 tensor-core MMA.
//
// The certificate and the reason no pivoting is needed are those of
// kernels_cert.cuh (nonsingular M-matrices with a relative row-dominance margin
// of kCertMargin and diagonal entries within [kCertDiagLo, kCertDiagHi]; the
// macro-atom matrices of calc_matom_matrix,
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

// RT: 64-row tiles one pass updates against the same R' tile (4 warps each);
// MINB: CTAs per SM asked of the register allocator
template <int RT_, int MINB_>
struct CgjlShape {
  static constexpr int RT = RT_;
  static constexpr int BT = 64;          // pivot columns per step; tile edge
  static constexpr int NTH = 128 * RT;   // 4 warps per row tile, a 2 x 2 grid of 32 x 32 sub-tiles
  static constexpr int SA = 68;          // shared tile row stride (doubles)
  static constexpr int MINB = MINB_;
  static constexpr int off_A = 0;                   // [RT][BT][SA] A operands: D^-1, or -W[I][K]
  static constexpr int off_B = RT * BT * SA;        // [BT][SA] B operand: W[K][J], or R'[K][J]
  static constexpr int off_x = (RT + 1) * BT * SA;  // [2][BT] pivot row, [2][BT] pivot column
  static constexpr int off_p = off_x + 4 * BT;      // [2] pivot reciprocals, by parity
  static constexpr int off_slot = off_p + 2;        // queue item broadcast
  static constexpr int n_dbl = off_slot + 2;
  static constexpr size_t dyn_smem = size_t(n_dbl) * 8;
  static_assert(RT == 1 || RT == 2, "one or two row tiles per pass");
  static_assert((NTH / 32) * (32 * 33) <= (RT + 1) * BT * SA, "running-total tiles fit the operand buffers");
  static_assert(dyn_smem <= 232448, "one CTA's shared memory");
};

namespace cgjl {

constexpr int BT = 64, SA = 68;
using Acc = double[4][4][2];

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// tile [r0, r0 + rb) x [c0, c0 + cb) of an n x n row-major matrix into a BT x BT
// shared tile, zero outside, negated when neg; NTH threads
template <int NTH>
__device__ __forceinline__ void load_tile(double* __restrict__ dst, const double* src, int n, int r0, int rb, int c0,
                                          int cb, bool neg, int tid) {
  constexpr int PER = BT * BT / NTH;
  double v[PER];
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int e = tid + NTH * m, r = e >> 6, c = e & 63;
    v[m] = (r < rb && c < cb) ? src[int64_t(r0 + r) * n + c0 + c] : 0.0;
  }
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int e = tid + NTH * m, r = e >> 6, c = e & 63;
    dst[r * SA + c] = neg ? -v[m] : v[m];
  }
}

template <int NTH>
__device__ __forceinline__ void identity_tile(double* __restrict__ dst, int rb, int tid) {
#pragma unroll
  for (int m = 0; m < BT * BT / NTH; ++m) {
    const int e = tid + NTH * m, r = e >> 6, c = e & 63;
    dst[r * SA + c] = (r == c && r < rb) ? 1.0 : 0.0;
  }
}

// a warp's 32 x 32 part of tile [r0 ..) x [c0 ..) in accumulator layout (lane:
// rows 8 i + g, columns 8 j + 2 t and + 1), zero outside or when zero; vec:
// rows start 16-byte aligned and n is even (each pair in or out together)
__device__ __forceinline__ void load_acc(Acc& acc, const double* src, int n, int r0, int rb, int c0, int cb,
                                         bool zero, bool vec, int wr, int wc, int g, int t) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = 32 * wr + 8 * i + g;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = 32 * wc + 8 * j + 2 * t;
      const double* a = src + int64_t(r0 + r) * n + c0 + c;
      if (vec) {
        const bool ok = !zero && r < rb && c < cb;
        const double2 v = ok ? *reinterpret_cast<const double2*>(a) : make_double2(0.0, 0.0);
        acc[i][j][0] = v.x;
        acc[i][j][1] = v.y;
      } else {
#pragma unroll
        for (int e = 0; e < 2; ++e) acc[i][j][e] = (!zero && r < rb && c + e < cb) ? a[e] : 0.0;
      }
    }
  }
}

// the same part written back, each entry times R[c0 + c] when R is set
__device__ __forceinline__ void store_acc(const Acc& acc, double* dst, int n, int r0, int rb, int c0, int cb,
                                          const double* __restrict__ R, bool vec, int wr, int wc, int g, int t) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = 32 * wr + 8 * i + g;
    if (r >= rb) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = 32 * wc + 8 * j + 2 * t;
      double* a = dst + int64_t(r0 + r) * n + c0 + c;
      double v0 = acc[i][j][0], v1 = acc[i][j][1];
      if (R) {
        if (c < cb) v0 = mul_rn(v0, __ldg(R + c0 + c));
        if (c + 1 < cb) v1 = mul_rn(v1, __ldg(R + c0 + c + 1));
      }
      if (vec) {
        if (c < cb) *reinterpret_cast<double2*>(a) = make_double2(v0, v1);
      } else {
        if (c < cb) a[0] = v0;
        if (c + 1 < cb) a[1] = v1;
      }
    }
  }
}

// rows [r0, r0 + rb) x columns [c0, c0 + cb) of an n x n row-major matrix
// brought into L2 (one prefetch per 16 doubles, every address inside the block)
__device__ __forceinline__ void prefetch_l2(const double* src, int n, int r0, int rb, int c0, int cb, int tid,
                                            int nth) {
  const int lpr = (cb + 15) >> 4;
  for (int e = tid; e < rb * lpr; e += nth) {
    const int r = e / lpr, l = e - r * lpr;
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(src + int64_t(r0 + r) * n + c0 + 16 * l));
  }
}

// acc += A B over the 64-deep tiles: warp (wr, wc) covers rows 32 wr .. +32,
// columns 32 wc .. +32 in 4 x 4 fragments
__device__ __forceinline__ void mma_tile(Acc& acc, const double* __restrict__ As, const double* __restrict__ Bs,
                                         int wr, int wc, int g, int t) {
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

// the same over a tile whose last rows, columns or depth are padding: only
// the kq 4-deep slices and this warp's ni x nj sub-blocks that hold data
__device__ __forceinline__ void mma_tile_edge(Acc& acc, const double* __restrict__ As,
                                              const double* __restrict__ Bs, int wr, int wc, int g, int t, int kq,
                                              int ni, int nj) {
  for (int kk = 0; kk < kq; ++kk) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = (i < ni) ? As[(32 * wr + 8 * i + g) * SA + 4 * kk + t] : 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = (j < nj) ? Bs[(4 * kk + t) * SA + 32 * wc + 8 * j + g] : 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (i < ni && j < nj) dmma_884(acc[i][j], a[i], b[j]);
  }
}

// acc += A B for a tile of rb rows, cb columns and depth kb
__device__ __forceinline__ void mma_any(Acc& acc, const double* __restrict__ As, const double* __restrict__ Bs,
                                        int wr, int wc, int g, int t, int rb, int cb, int kb) {
  if (rb == BT && cb == BT && kb == BT) {
    mma_tile(acc, As, Bs, wr, wc, g, t);
  } else {
    const int ni = min(4, max(0, (rb - 32 * wr + 7) >> 3)), nj = min(4, max(0, (cb - 32 * wc + 7) >> 3));
    if (ni > 0 && nj > 0) mma_tile_edge(acc, As, Bs, wr, wc, g, t, (kb + 3) >> 2, ni, nj);
  }
}

}  // namespace cgjl

template <int RT, int MINB>
__global__ void __launch_bounds__(128 * RT, MINB)
    cgjl_inverse_kernel(BatchView bv, CertArgs ca, CertEpi ep, int* __restrict__ queue) {
  using namespace cgjl;
  using S = CgjlShape<RT, MINB>;
  constexpr int NTH = S::NTH, NWARP = NTH / 32;
  constexpr int RPT = BT / (NTH / 64);   // rows of the pivot block per thread in the D^-1 phase
  extern __shared__ __align__(16) double sm[];
  double* As = sm + S::off_A;
  double* Bs = sm + S::off_B;
  double* xr = sm + S::off_x;       // pivot rows, by parity of the pivot
  double* xc = xr + 2 * BT;         // pivot columns, by parity
  int* slot = reinterpret_cast<int*>(sm + S::off_slot);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int rt = warp >> 2;                       // the row tile of this warp's pass
  const int wr = (warp >> 1) & 1, wc = warp & 1;  // its 32 x 32 part
  const double* Ao = As + rt * (BT * SA);         // its A operand
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
    const bool vA = ((n & 1) == 0) && ((reinterpret_cast<uintptr_t>(Ag) & 15) == 0);
    const bool vW = ((n & 1) == 0) && ((reinterpret_cast<uintptr_t>(Wg) & 15) == 0);

    // ---- certificate, a warp per row, all of a row's loads in flight at once
    bool ok = true;
    for (int r = warp; r < n; r += NWARP) {
      const double* row = Ag + int64_t(r) * n;
      double v[32];
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        const int c = lane + 32 * u;
        v[u] = (c < n) ? row[c] : 0.0;
      }
      const double d = row[r];
      double off = 0.0;
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        const int c = lane + 32 * u;
        if (c != r) {
          ok &= (v[u] <= 0.0);   // false for NaN
          off += fabs(v[u]);
        }
      }
      off = warp_sum(off);
      ok &= (d >= kCertDiagLo) && (d <= kCertDiagHi) && (off * (1.0 + 0x1p-40) <= (1.0 - kCertMargin) * d);
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
      const bool vs = (kt == 0) ? vA : vW;

      // ---- D^-1 into As[0]: thread (column c, rows RPT h ..) of the padded block
      {
        const int c = tid & 63, h = tid >> 6;
        double dv[RPT];
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
          const int r = RPT * h + i;
          dv[i] = (r < kb && c < kb) ? src[int64_t(k0 + r) * n + k0 + c] : (r == c ? 1.0 : 0.0);
        }
        double* px = sm + S::off_p;
        // pivot j = RPT jh + jj: the holder of the pivot entry forms its
        // reciprocal once; the holders of row j and column j publish them
        for (int jh = 0; jh < BT / RPT; ++jh) {
#pragma unroll
          for (int jj = 0; jj < RPT; ++jj) {
            const int j = RPT * jh + jj, par = jj & 1;
            double* rx = xr + par * BT;
            double* cx = xc + par * BT;
            if (h == jh) {
              rx[c] = dv[jj];
              if (c == j) px[par] = 1.0 / dv[jj];
            }
            if (c == j) {
#pragma unroll
              for (int i = 0; i < RPT; ++i) cx[RPT * h + i] = dv[i];
            }
            __syncthreads();
            const double p = px[par];
            const double rj = rx[c] * p;
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
              if (h == jh && i == jj) {
                dv[i] = (c == j) ? p : rj;
              } else {
                const double f = cx[RPT * h + i];
                dv[i] = (c == j) ? -f * p : fma(-f, rj, dv[i]);
              }
            }
          }
        }
#pragma unroll
        for (int i = 0; i < RPT; ++i) As[(RPT * h + i) * SA + c] = dv[i];
      }

      // ---- R' = D^-1 W[K][J] on the pivot rows (D^-1 on K's own tile); with
      // two row groups, the second takes tile J + 1 with its B operand in As[1]
      for (int jt = 0; jt < nb; jt += RT) {
        __syncthreads();   // D^-1 written / the previous tiles' operands read
#pragma unroll
        for (int q = 0; q < RT; ++q) {
          const int jq = jt + q;
          double* Bq = (q == 0) ? Bs : As + BT * SA;
          if (jq < nb) {
            if (jq == kt) identity_tile<NTH>(Bq, kb, tid);
            else load_tile<NTH>(Bq, src, n, k0, kb, jq * BT, min(BT, n - jq * BT), false, tid);
          }
        }
        __syncthreads();
        const int jq = jt + rt;
        if (jq < nb) {
          Acc acc;
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
          mma_any(acc, As, (rt == 0) ? Bs : As + BT * SA, wr, wc, g, t, kb, min(BT, n - jq * BT), kb);
          // the pivot rows stay unscaled by R until no tile reads them
          store_acc(acc, Wg, n, k0, kb, jq * BT, min(BT, n - jq * BT), nullptr, vW, wr, wc, g, t);
        }
      }
      __syncthreads();

      // ---- the other row tiles, RT per pass: W[I][:] += (-W[I][K]) R'
      const bool last = (kt == nb - 1);
      const double* __restrict__ Rs = (last && ep.R) ? ep.R + ep.offv[s] : nullptr;
      for (int ip = 0; ip < nb - 1; ip += RT) {
        // pass rows: the ip-th .. other-than-K row tiles
        auto tile_row = [&](int u) { return u + (u >= kt); };
#pragma unroll
        for (int q = 0; q < RT; ++q) {
          const int u = ip + q;
          if (u < nb - 1) {
            const int i0 = tile_row(u) * BT;
            load_tile<NTH>(As + q * (BT * SA), src, n, i0, min(BT, n - i0), k0, kb, true, tid);
          }
        }
        const int u = ip + rt;
        const bool act = u < nb - 1;
        const int i0 = act ? tile_row(u) * BT : 0, ib = act ? min(BT, n - i0) : 0;
        for (int jt = 0; jt < nb; ++jt) {
          const int j0 = jt * BT, jb = min(BT, n - j0);
          // the tile's own values first (HBM), then R' (L2): both in flight at once
          Acc acc;
          load_acc(acc, src, n, i0, ib, j0, jb, jt == kt || !act, vs, wr, wc, g, t);
          load_tile<NTH>(Bs, Wg, n, k0, kb, j0, jb, false, tid);
          __syncthreads();
          // the next tile's operands (or the next pass's column strips and
          // first tile) are brought into L2 while this tile's MMAs run
          if (jt + 1 < nb) {
            const int j1 = (jt + 1) * BT, jb1 = min(BT, n - j1);
            prefetch_l2(Wg, n, k0, kb, j1, jb1, tid, NTH);
            if (jt + 1 != kt) {
#pragma unroll
              for (int q = 0; q < RT; ++q) {
                const int uq = ip + q;
                if (uq < nb - 1) {
                  const int iq = tile_row(uq) * BT;
                  prefetch_l2(src, n, iq, min(BT, n - iq), j1, jb1, tid, NTH);
                }
              }
            }
          } else {
#pragma unroll
            for (int q = 0; q < RT; ++q) {
              const int uq = ip + RT + q;
              if (uq < nb - 1) {
                const int iq = tile_row(uq) * BT, ibq = min(BT, n - iq);
                prefetch_l2(src, n, iq, ibq, k0, kb, tid, NTH);
                if (kt != 0) prefetch_l2(src, n, iq, ibq, 0, min(BT, n), tid, NTH);
              }
            }
            prefetch_l2(Wg, n, k0, kb, 0, min(BT, n), tid, NTH);
          }
          if (act) {
            mma_any(acc, Ao, Bs, wr, wc, g, t, ib, jb, kb);
            store_acc(acc, Wg, n, i0, ib, j0, jb, Rs, vW, wr, wc, g, t);
          }
          __syncthreads();
        }
      }
      // the pivot rows of the last step, scaled now that no tile reads them
      if (Rs) {
        for (int e = tid; e < kb * n; e += NTH) {
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
      for (int r0 = 32 * warp; r0 < n; r0 += 32 * NWARP) {
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
