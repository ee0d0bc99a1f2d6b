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
  static constexpr int n_dbl0 = off_S + 2 * B;
  static constexpr int n_dbl = n_dbl0 > P * LS ? n_dbl0 : P * LS;
  static constexpr int n_int = 5 * P + 8;  // ipiv, perm, slot_src, slot_dst, total, flags
  static constexpr int PER = (P * P + NT - 1) / NT;   // staged elements per thread
  static constexpr size_t panel_bytes = size_t(n_dbl) * 8 + size_t(n_int) * 4;
  static constexpr size_t lu_bytes = size_t(P) * LS * 8 + size_t(2 * P) * 8 + size_t(P) * 4;
  // the whole matrix passes through shared memory (row stride LS) on its way
  // in and out, so the global loads and stores are row-coalesced
  static constexpr size_t stage_bytes = size_t(P) * LS * 8;
  static constexpr size_t dyn_smem_a = (KIND == kSolve && lu_bytes > panel_bytes) ? lu_bytes : panel_bytes;
  static constexpr size_t dyn_smem = dyn_smem_a > stage_bytes + size_t(n_int) * 4 + 64 ? dyn_smem_a : stage_bytes + size_t(n_int) * 4 + 64;
  static constexpr int regs = 72 + 5 * B * B / 2;
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
  int* total = slot_dst + P;             // [P] original row now at each row (GSL's permutation)
  int* flags = total + P;                // [0] singular

  const int t = threadIdx.x;
  const int tr = t / TG, tc = t % TG;
  const int row0 = tr * B, col0 = tc * B;
  const int wid = t >> 5, wl = t & 31;

  for (int item = blockIdx.x; item < bv.count; item += gridDim.x) {
    const int s = bv.list[item];
    const int n = bv.n[s];
    const double* __restrict__ Ag = bv.A + bv.offA[s];

    // coalesced load of the padded P x P matrix, every load of a thread in
    // flight at once, through shared memory to the register blocks
    {
      double* stage = dsm;
      double v[Sh::PER];
#pragma unroll
      for (int u = 0; u < Sh::PER; ++u) {
        const int e = t + u * Sh::NT, row = e / P, col = e - (e / P) * P;
        v[u] = (e < P * P && row < n && col < n) ? __ldg(Ag + int64_t(row) * n + col) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < Sh::PER; ++u) {
        const int e = t + u * Sh::NT, row = e / P, col = e - (e / P) * P;
        if (e < P * P) stage[row * Sh::LS + col] = v[u];
      }
      if (t < P) total[t] = t;
      __syncthreads();
    }
    double a[B][B];
#pragma unroll
    for (int r = 0; r < B; ++r)
#pragma unroll
      for (int c = 0; c < B; ++c) a[r][c] = dsm[(row0 + r) * Sh::LS + col0 + c];
    __syncthreads();
    if (t == 0) flags[0] = 0;

    const int npan = (n + B - 1) / B;
    for (int jb = 0; jb < npan; ++jb) {
      const int j0 = jb * B;
      const int nb = min(B, n - j0);
      // ---- 1. panel to shared memory, per-panel bookkeeping reset ----------
      if (t < P) { slot_src[t] = -1; slot_dst[t] = -1; perm[t] = t; }
      if (t < B) rinv_s[t] = 0.0;     // padding steps of the last panel contribute nothing
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

      // ---- 2. warp 0 factorises the panel in its registers -----------------
      // Lane l holds panel rows l, l+32, ... (indexed by the row they had when
      // the panel started); rows keep their place and carry their current
      // position, so ties break as GSL's physical swaps would.  Multipliers and
      // the factorised panel are stored by that origin row; perm[q] = origin of
      // the row that ends at position q.
      if (wid == 0) {
        constexpr int RPL = (P + 31) / 32;
        double pr[RPL][B];
        int ps[RPL];
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          const int r = wl + 32 * i;
          ps[i] = r;
#pragma unroll
          for (int c = 0; c < B; ++c) pr[i][c] = (r < n) ? Pn[r * PS + c] : 0.0;
        }
        bool sing = false;
#pragma unroll
        for (int k = 0; k < B; ++k) {
          if (k < nb && !sing) {
            const int j = j0 + k;
            double bk = -1.0;
            int bp = 0x7fffffff, bw = 0;
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
              const int r = wl + 32 * i;
              if (r < n && ps[i] >= j) {
                const double key = pivot_key(pr[i][k]);
                if (pivot_better(key, ps[i], bk, bp)) { bk = key; bp = ps[i]; bw = (wl << 3) | i; }
              }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
              const double ok = __shfl_xor_sync(0xffffffffu, bk, off);
              const int op = __shfl_xor_sync(0xffffffffu, bp, off);
              const int ow = __shfl_xor_sync(0xffffffffu, bw, off);
              if (pivot_better(ok, op, bk, bp)) { bk = ok; bp = op; bw = ow; }
            }
            const int pl = bw >> 3, pi = bw & 7, ppos = bp;
            if (wl == 0) ipiv[j] = ppos;
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
              if (wl == pl && i == pi) ps[i] = j;
              else if (ps[i] == j) ps[i] = ppos;
            }
            double pv[B];
#pragma unroll
            for (int c = 0; c < B; ++c) {
              double mine = pr[0][c];
#pragma unroll
              for (int i = 1; i < RPL; ++i) mine = (pi == i) ? pr[i][c] : mine;
              pv[c] = __shfl_sync(0xffffffffu, mine, pl);
            }
            const double ujj = pv[k];
            if (ujj == 0.0) {
              sing = true;
            } else {
              const double rinv = __drcp_rn(ujj);   // correctly rounded, = fl(1/ujj)
#pragma unroll
              for (int i = 0; i < RPL; ++i) {
                const int r = wl + 32 * i;
                const bool is_piv = (wl == pl) && (i == pi);
                if (r < n && !is_piv) {
                  const bool below = ps[i] > j;
                  if (KIND == kInvert || below) {
                    const double l = below ? gsl_multiplier(pr[i][k], ujj, rinv) : mul_rn(pr[i][k], rinv);
                    Mm[r * PS + k] = l;
#pragma unroll
                    for (int c = 0; c < B; ++c) {
                      if (c == k || (KIND == kSolve && c < k)) continue;
                      pr[i][c] = sub_rn(pr[i][c], mul_rn(l, pv[c]));
                    }
                    pr[i][k] = (KIND == kInvert) ? -l : l;
                  }
                }
                if (KIND == kInvert && is_piv) {
#pragma unroll
                  for (int c = 0; c < B; ++c) pr[i][c] = (c == k) ? rinv : mul_rn(pr[i][c], rinv);
                }
              }
              if (wl == 0) rinv_s[k] = rinv;
            }
          }
        }
        if (sing) {
          if (wl == 0) flags[0] = 1;
        } else {
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const int r = wl + 32 * i;
            if (r < n) {
#pragma unroll
              for (int c = 0; c < B; ++c) Pn[r * PS + c] = pr[i][c];
              perm[ps[i]] = r;
            }
          }
          __syncwarp();
          // staging slots of the rows whose content changes
          int base = 0;
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const int q = wl + 32 * i;
            const bool moved = (q < n) && (perm[q] != q);
            const unsigned mask = __ballot_sync(0xffffffffu, moved);
            if (moved) {
              const int sl = base + __popc(mask & ((1u << wl) - 1u));
              slot_dst[q] = sl;
              slot_src[perm[q]] = sl;
            }
            base += __popc(mask);
          }
        }
      }
      __syncthreads();
      if (flags[0]) break;

      // ---- 3. the panel's row swaps on the other columns ------------------
      int tot_new = 0;
      if (t < P) tot_new = total[perm[t]];
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
      if (t < P) total[t] = tot_new;
      if (tc != jb) {
#pragma unroll
        for (int r = 0; r < B; ++r) {
          const int sl = slot_dst[row0 + r];
          if (sl >= 0) {
#pragma unroll
            for (int c = 0; c < B; ++c) a[r][c] = Rs[sl * P + col0 + c];
          }
        }
        // ---- 4. pivot rows at their own step (thread row jb), in registers -
        if (tr == jb && (KIND == kInvert || tc > jb)) {
          // padding rows of a last, partial panel are zero with zero multipliers,
          // so every loop runs over the full panel width
#pragma unroll
          for (int k = 1; k < B; ++k) {
            const int org = perm[j0 + k];
            double mk[B];
#pragma unroll
            for (int kk = 0; kk < k; ++kk) mk[kk] = Mm[org * PS + kk];
#pragma unroll
            for (int c = 0; c < B; ++c) {
              double v = a[k][c];
#pragma unroll
              for (int kk = 0; kk < k; ++kk) v = sub_rn(v, mul_rn(mk[kk], a[kk][c]));
              a[k][c] = v;
            }
          }
#pragma unroll
          for (int k = 0; k < B; ++k)
#pragma unroll
            for (int c = 0; c < B; ++c) Vs[k * P + col0 + c] = a[k][c];
        }
      }
      __syncthreads();

      // ---- 5. rank-nb update of this thread's block ------------------------
      if (tc == jb) {
#pragma unroll
        for (int r = 0; r < B; ++r) {
          const int org = perm[row0 + r];
#pragma unroll
          for (int c = 0; c < B; ++c) a[r][c] = Pn[org * PS + c];
        }
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
                  const int org = perm[j0 + k];
                  acc = acc * rinv_s[k];
#pragma unroll
                  for (int k2 = k + 1; k2 < B; ++k2)
                    if (k2 < nb) acc = fma(-Mm[org * PS + k2], Vs[k2 * P + col0 + c], acc);
                }
                a[k][c] = acc;
              }
            }
          }
        }
      } else {
        const bool lu_region = (tr > jb) && (tc > jb);   // below the panel, right of it
        int org[B];
#pragma unroll
        for (int r = 0; r < B; ++r) org[r] = perm[row0 + r];
        if (lu_region) {
          // GSL's LU region: one rounding per product and per difference, k ascending
#pragma unroll
          for (int k = 0; k < B; ++k) {
            double vk[B], mk[B];
#pragma unroll
            for (int c = 0; c < B; ++c) vk[c] = Vs[k * P + col0 + c];
#pragma unroll
            for (int r = 0; r < B; ++r) mk[r] = Mm[org[r] * PS + k];
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
              for (int c = 0; c < B; ++c) a[r][c] = sub_rn(a[r][c], mul_rn(mk[r], vk[c]));
          }
        } else if (KIND == kInvert) {
          // rows above the panel or columns left of it: outside the LU region
#pragma unroll
          for (int k = 0; k < B; ++k) {
            double vk[B], mk[B];
#pragma unroll
            for (int c = 0; c < B; ++c) vk[c] = Vs[k * P + col0 + c];
#pragma unroll
            for (int r = 0; r < B; ++r) mk[r] = Mm[org[r] * PS + k];
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
              for (int c = 0; c < B; ++c) a[r][c] = fma(-mk[r], vk[c], a[r][c]);
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
      // A^-1 = W P: output column total[i] takes column i of W
      double* stage = dsm;
#pragma unroll
      for (int r = 0; r < B; ++r) {
        const int row = row0 + r;
        if (row < n) {
#pragma unroll
          for (int c = 0; c < B; ++c) {
            const int col = col0 + c;
            if (col < n) stage[row * Sh::LS + total[col]] = a[r][c];
          }
        }
      }
      __syncthreads();
      double* __restrict__ Og = bv.out + bv.offA[s];
#pragma unroll
      for (int u = 0; u < Sh::PER; ++u) {
        const int e = t + u * Sh::NT, row = e / P, col = e - (e / P) * P;
        if (e < P * P && row < n && col < n) Og[int64_t(row) * n + col] = stage[row * Sh::LS + col];
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
      // GSL's permutation (lu.c:95-109): pm[i] = original row now at i
      if (t < n) pm[t] = total[t];
      __syncthreads();
#pragma unroll
      for (int r = 0; r < B; ++r)
#pragma unroll
        for (int c = 0; c < B; ++c) lu[(row0 + r) * LS + col0 + c] = a[r][c];
      __syncthreads();
      if (wid == 0) {
        const int64_t ov = bv.offv[s];
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
