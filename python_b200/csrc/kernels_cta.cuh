// CTA-per-system kernels for 32 < n <= 128 (macro-atom jumping matrices of a
// few dozen levels, per-element macro populations).
//
// The padded P x P matrix lives in registers: a TG x TG thread grid, thread
// (tr, tc) owning the B x B block of rows [tr*B, tr*B+B) and columns
// [tc*B, tc*B+B).  The factorisation is blocked by panels of B columns, so the
// panel of block column jb is exactly thread column jb and its pivot rows are
// exactly thread row jb; every register index is a compile-time constant.
// Per panel:
//   1. the panel's owners copy it (all rows) to shared memory;
//   2. warp 0 factorises the n x B panel there with physical row swaps, as
//      GSL's LU_decomp_L2 does on a panel (lu.c:129-191): first strict maximum
//      pivot, multipliers a * fl(1/u) (a / u below DBL_MIN), each update one
//      rounding per product and per difference; every row's multipliers are
//      recorded (M, n x B);
//   3. the panel's row swaps are applied to the other columns (apply_pivots,
//      lu.c:263) by moving the affected rows through shared memory;
//   4. thread row jb rebuilds the pivot rows' values at their own step,
//      V_k = W_k - sum_{k'<k} M[k][k'] V_k' (the dtrsm of lu.c:266);
//   5. every other block takes W -= M V with k ascending (the dgemm of lu.c:269).
// Every entry of the LU region therefore sees GSL's operation sequence.  For an
// inverse the same sweep is an in-place Gauss-Jordan: rows above the panel and
// columns left of it are eliminated too (fused multiply-add is allowed there,
// outside the LU region), pivot rows are scaled by 1/u_kk, and the columns are
// unscrambled in reverse pivot order at the end.  A solve keeps the LU factors
// and runs LU_svx's triangular sweeps in GSL's order from shared memory.
#pragma once
#include "ss_common.cuh"

namespace ss {

template <int KIND, int TG, int B>
struct CtaShape {
  static constexpr int P = TG * B;         // padded order
  static constexpr int NT = TG * TG;       // threads
  static constexpr int NW = NT / 32;
  static constexpr int PS = B + 1;         // panel row stride (odd)
  static constexpr int LS = P + 1;         // LU row stride for the solve sweeps
  // shared-memory layout (doubles): panel, multipliers, V, moved rows, scalars
  static constexpr int off_M = P * PS;
  static constexpr int off_V = 2 * P * PS;
  static constexpr int off_R = off_V + B * P;
  static constexpr int off_S = off_R + 2 * B * P;
  static constexpr int n_dbl = off_S + 2 * B;
  static constexpr int n_int = 4 * P + 8;  // ipiv, perm, slot_src, slot_dst, flags
  static constexpr size_t panel_bytes = size_t(n_dbl) * 8 + size_t(n_int) * 4;
  static constexpr size_t lu_bytes = size_t(P) * LS * 8 + size_t(2 * P) * 8 + size_t(P) * 4;
  static constexpr size_t dyn_smem = (KIND == kSolve && lu_bytes > panel_bytes) ? lu_bytes : panel_bytes;
  static constexpr int regs = 56 + 5 * B * B / 2;
  static constexpr int min_blocks = (65536 / (NT * (regs > 255 ? 255 : regs))) < 1
                                        ? 1 : (65536 / (NT * (regs > 255 ? 255 : regs)));
  static_assert(NT % 32 == 0, "whole warps");
  static_assert(NT >= P, "one thread per row for the per-panel resets");
};

template <int KIND, int TG, int B>
__global__ void __launch_bounds__(TG * TG, (CtaShape<KIND, TG, B>::min_blocks))
cta_exact_kernel(BatchView bv) {
  using Sh = CtaShape<KIND, TG, B>;
  constexpr int P = Sh::P;
  constexpr int PS = Sh::PS;
  extern __shared__ __align__(16) double dsm[];
  double* Pn = dsm;                      // [P][PS] panel
  double* Mm = dsm + Sh::off_M;          // [P][PS] multipliers of this panel
  double* Vs = dsm + Sh::off_V;          // [B][P]  pivot rows at their step
  double* Rs = dsm + Sh::off_R;          // [2B][P] rows moved by the swaps
  double* rinv_s = dsm + Sh::off_S;      // [B]
  int* ipiv = reinterpret_cast<int*>(dsm + Sh::n_dbl);   // [P]
  int* perm = ipiv + P;                  // [P] source row of each row after this panel's swaps
  int* slot_src = perm + P;              // [P] staging slot of a row that moves, -1 otherwise
  int* slot_dst = slot_src + P;          // [P] staging slot a row is refilled from, -1 otherwise
  int* flags = slot_dst + P;             // [0] singular

  const int t = threadIdx.x;
  const int tr = t / TG, tc = t % TG;
  const int row0 = tr * B, col0 = tc * B;
  const int wid = t >> 5, wl = t & 31;

  for (int item = blockIdx.x; item < bv.count; item += gridDim.x) {
    const int s = bv.list[item];
    const int n = bv.n[s];
    const double* __restrict__ Ag = bv.A + bv.offA[s];

    double a[B][B];
#pragma unroll
    for (int r = 0; r < B; ++r) {
      const int row = row0 + r;
#pragma unroll
      for (int c = 0; c < B; ++c) {
        const int col = col0 + c;
        a[r][c] = (row < n && col < n) ? __ldg(Ag + int64_t(row) * n + col) : 0.0;
      }
    }
    if (t == 0) flags[0] = 0;

    const int npan = (n + B - 1) / B;
    for (int jb = 0; jb < npan; ++jb) {
      const int j0 = jb * B;
      const int nb = min(B, n - j0);
      // ---- 1. panel to shared memory, per-panel bookkeeping reset ----------
      if (t < P) { slot_src[t] = -1; slot_dst[t] = -1; perm[t] = t; }
      if (tc == jb) {
#pragma unroll
        for (int r = 0; r < B; ++r)
#pragma unroll
          for (int c = 0; c < B; ++c) {
            Pn[(row0 + r) * PS + c] = a[r][c];
            Mm[(row0 + r) * PS + c] = 0.0;
          }
      }
      __syncthreads();

      // ---- 2. warp 0 factorises the panel --------------------------------
      if (wid == 0) {
        for (int k = 0; k < nb; ++k) {
          const int j = j0 + k;
          double bk = -1.0;
          int br = 0x7fffffff;
          for (int r = j + wl; r < n; r += 32) {
            const double key = pivot_key(Pn[r * PS + k]);
            if (pivot_better(key, r, bk, br)) { bk = key; br = r; }
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            const double ok = __shfl_xor_sync(0xffffffffu, bk, off);
            const int orr = __shfl_xor_sync(0xffffffffu, br, off);
            if (pivot_better(ok, orr, bk, br)) { bk = ok; br = orr; }
          }
          const int p = br;
          if (wl == 0) ipiv[j] = p;
          if (p != j && wl < B) {
            const double x = Pn[j * PS + wl]; Pn[j * PS + wl] = Pn[p * PS + wl]; Pn[p * PS + wl] = x;
            const double y = Mm[j * PS + wl]; Mm[j * PS + wl] = Mm[p * PS + wl]; Mm[p * PS + wl] = y;
          }
          __syncwarp();
          const double ujj = Pn[j * PS + k];
          if (ujj == 0.0) {
            if (wl == 0) flags[0] = 1;
            break;
          }
          const double rinv = __drcp_rn(ujj);   // correctly rounded, = fl(1/ujj)
          double piv[B];
#pragma unroll
          for (int c = 0; c < B; ++c) piv[c] = Pn[j * PS + c];
          __syncwarp();
          for (int r = wl; r < n; r += 32) {
            if (r == j) continue;
            if (KIND == kSolve && r < j) continue;
            const double v = Pn[r * PS + k];
            const double l = (r > j) ? gsl_multiplier(v, ujj, rinv) : mul_rn(v, rinv);
            Mm[r * PS + k] = l;
#pragma unroll
            for (int c = 0; c < B; ++c) {
              if (c == k || c >= nb) continue;
              if (KIND == kSolve && c < k) continue;
              Pn[r * PS + c] = sub_rn(Pn[r * PS + c], mul_rn(l, piv[c]));
            }
            Pn[r * PS + k] = (KIND == kInvert) ? -l : l;
          }
          if (wl == 0) {
            rinv_s[k] = rinv;
            if (KIND == kInvert) {
#pragma unroll
              for (int c = 0; c < B; ++c) Pn[j * PS + c] = (c == k) ? rinv : mul_rn(piv[c], rinv);
            }
          }
          __syncwarp();
        }
        if (wl == 0 && flags[0] == 0) {
          // net row permutation of this panel and the staging slots of moved rows
          for (int k = 0; k < nb; ++k) {
            const int q = ipiv[j0 + k];
            if (q != j0 + k) { const int x = perm[j0 + k]; perm[j0 + k] = perm[q]; perm[q] = x; }
          }
          int m = 0;
          for (int k = 0; k < nb; ++k) {
            const int q = ipiv[j0 + k];
            if (q == j0 + k) continue;
            const int cand[2] = {j0 + k, q};
            for (int ci = 0; ci < 2; ++ci) {
              const int rr = cand[ci];
              if (perm[rr] != rr && slot_dst[rr] < 0) {
                slot_dst[rr] = m;
                slot_src[perm[rr]] = m;
                ++m;
              }
            }
          }
        }
      }
      __syncthreads();
      if (flags[0]) break;

      // ---- 3. the panel's row swaps on the other columns ------------------
      if (tc != jb) {
#pragma unroll
        for (int r = 0; r < B; ++r) {
          const int sl = slot_src[row0 + r];
          if (sl >= 0) {
#pragma unroll
            for (int c = 0; c < B; ++c) Rs[sl * P + col0 + c] = a[r][c];
          }
        }
      }
      __syncthreads();
      if (tc != jb) {
#pragma unroll
        for (int r = 0; r < B; ++r) {
          const int sl = slot_dst[row0 + r];
          if (sl >= 0) {
#pragma unroll
            for (int c = 0; c < B; ++c) a[r][c] = Rs[sl * P + col0 + c];
          }
        }
        // ---- 4. pivot rows at their own step (thread row jb) --------------
        if (tr == jb && (KIND == kInvert || tc > jb)) {
#pragma unroll
          for (int k = 0; k < B; ++k) {
            if (k < nb) {
#pragma unroll
              for (int c = 0; c < B; ++c) {
                double v = a[k][c];
#pragma unroll
                for (int kk = 0; kk < k; ++kk)
                  v = sub_rn(v, mul_rn(Mm[(j0 + k) * PS + kk], Vs[kk * P + col0 + c]));
                Vs[k * P + col0 + c] = v;
              }
            }
          }
        }
      }
      __syncthreads();

      // ---- 5. rank-nb update of this thread's block ------------------------
      if (tc == jb) {
#pragma unroll
        for (int r = 0; r < B; ++r)
#pragma unroll
          for (int c = 0; c < B; ++c) a[r][c] = Pn[(row0 + r) * PS + c];
      } else if (tr == jb) {
        // the panel's pivot rows: their final values from V
        if (KIND == kInvert || tc > jb) {
#pragma unroll
          for (int k = 0; k < B; ++k) {
            if (k < nb) {
#pragma unroll
              for (int c = 0; c < B; ++c) {
                double acc = Vs[k * P + col0 + c];
                if (KIND == kInvert) {
                  acc = acc * rinv_s[k];
#pragma unroll
                  for (int k2 = k + 1; k2 < B; ++k2)
                    if (k2 < nb) acc = fma(-Mm[(j0 + k) * PS + k2], Vs[k2 * P + col0 + c], acc);
                }
                a[k][c] = acc;
              }
            }
          }
        }
      } else {
        const bool lu_region = (tr > jb) && (tc > jb);   // below the panel, right of it
        if (KIND == kInvert || lu_region) {
#pragma unroll
          for (int k = 0; k < B; ++k) {
            if (k < nb) {
              double vk[B];
#pragma unroll
              for (int c = 0; c < B; ++c) vk[c] = Vs[k * P + col0 + c];
#pragma unroll
              for (int r = 0; r < B; ++r) {
                const double m = Mm[(row0 + r) * PS + k];
                if (lu_region) {
#pragma unroll
                  for (int c = 0; c < B; ++c) a[r][c] = sub_rn(a[r][c], mul_rn(m, vk[c]));
                } else {
#pragma unroll
                  for (int c = 0; c < B; ++c) a[r][c] = fma(-m, vk[c], a[r][c]);
                }
              }
            }
          }
        }
      }
      __syncthreads();
    }

    if (flags[0]) {
      if (t == 0) {
        bv.status[s] = (KIND == kSolve) ? kSolveSingular : kInvertSingular;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
      __syncthreads();
      continue;
    }

    if (KIND == kInvert) {
      // reverse-order column unscramble: output column perm[k] takes column k
      if (t == 0) {
        int* src = slot_src;
        for (int c = 0; c < n; ++c) src[c] = c;
        for (int jj = n - 1; jj >= 0; --jj) {
          const int q = ipiv[jj];
          if (q != jj) { const int x = src[jj]; src[jj] = src[q]; src[q] = x; }
        }
        for (int c = 0; c < n; ++c) perm[src[c]] = c;
      }
      __syncthreads();
      double* __restrict__ Og = bv.out + bv.offA[s];
#pragma unroll
      for (int r = 0; r < B; ++r) {
        const int row = row0 + r;
        if (row < n) {
#pragma unroll
          for (int c = 0; c < B; ++c) {
            const int col = col0 + c;
            if (col < n) Og[int64_t(row) * n + perm[col]] = a[r][c];
          }
        }
      }
      if (t == 0) {
        bv.status[s] = kOk;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
    } else {
      // LU (rows already in GSL's order) into shared memory for the sweeps;
      // the pivots survive in ipiv, which the LU copy does not overlap
      constexpr int LS = Sh::LS;
      double* lu = dsm;
      double* vec = dsm + P * LS;
      double* xs = vec + P;
      int* pm = reinterpret_cast<int*>(xs + P);
      // the pivots sit inside the area the LU copy overwrites: move them first
      if (t < n) pm[t] = ipiv[t];
      __syncthreads();
#pragma unroll
      for (int r = 0; r < B; ++r)
#pragma unroll
        for (int c = 0; c < B; ++c) lu[(row0 + r) * LS + col0 + c] = a[r][c];
      __syncthreads();
      if (wid == 0) {
        const int64_t ov = bv.offv[s];
        // gsl_permutation from the row swaps (lu.c:95-109), built in place of
        // the pivots: pm[i] = original row now at i
        if (wl == 0) {
          int* sw = reinterpret_cast<int*>(vec);   // scratch copy of the pivots
          for (int i = 0; i < n; ++i) sw[i] = pm[i];
          for (int i = 0; i < n; ++i) pm[i] = i;
          for (int i = 0; i < n; ++i) {
            const int q = sw[i];
            if (pm[q] != pm[i]) { const int x = pm[q]; pm[q] = pm[i]; pm[i] = x; }
          }
        }
        __syncwarp();
        for (int i = wl; i < n; i += 32) vec[i] = bv.b[ov + pm[i]];
        __syncwarp();
        // forward sweep (unit L), ascending j per entry
        for (int j = 0; j < n; ++j) {
          const double yj = vec[j];
          for (int i = j + 1 + wl; i < n; i += 32) vec[i] = sub_rn(vec[i], mul_rn(lu[i * LS + j], yj));
          __syncwarp();
        }
        // backward sweep in LU_svx's order (serial chain)
        if (wl == 0) {
          for (int i = n - 1; i >= 0; --i) {
            double u = vec[i];
            for (int k = i + 1; k < n; ++k) u = sub_rn(u, mul_rn(lu[i * LS + k], xs[k]));
            xs[i] = div_rn(u, lu[i * LS + i]);
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
