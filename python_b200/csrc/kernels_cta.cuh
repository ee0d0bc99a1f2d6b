// CTA-per-system kernels for 32 < n <= 160 (macro-atom jumping matrices of a
// few dozen to ~160 levels, per-element macro populations).
//
// The padded P x P matrix stays in shared memory for the whole factorisation
// (row-major, columns XOR-swizzled inside 16-column groups so that row, column
// and tile accesses are all free of bank conflicts).  Rows never move: each
// physical row carries its current position (ps), and perm[q] names the row
// at position q, so GSL's row swaps cost two integer stores and ties in the
// pivot search break on positions exactly as GSL's physical swaps would.
// The factorisation is blocked by panels of B = 8 columns.  Per panel:
//   1. warp 0 factorises the n x B panel in its registers (GSL's LU_decomp_L2
//      on a panel, lu.c:129-191): first strict maximum pivot by a three-step
//      warp reduction of (|a|, position), multipliers a * fl(1/u) (a / u below
//      DBL_MIN), one rounding per product and per difference; every row's
//      multipliers are recorded (Mm);
//   2. one thread per column rebuilds the panel's pivot rows at their own step,
//      V_k = W_k - sum_{k'<k} Mm[k][k'] V_k' (the dtrsm of lu.c:266);
//   3. every thread updates its tile, W -= Mm V with k ascending (the dgemm
//      of lu.c:269), one rounding per product and per difference.
// Every entry of the LU region therefore sees GSL's operation sequence.  For an
// inverse the same sweep is an in-place Gauss-Jordan: rows above the panel and
// columns left of it are eliminated too, pivot rows are scaled by 1/u_kk, and
// the result is read out through the row and column permutations.  A solve
// keeps the LU factors and runs LU_svx's triangular sweeps in GSL's order.
#pragma once
#include "ss_common.cuh"

namespace ss {

// Column swizzle of row r: bit 3 alternates with the row's parity and bits 0-2
// take the next three row bits, so 32 consecutive rows of one column, and
// 4 consecutive rows x 8 consecutive columns, both hit every bank pair twice.
__device__ __forceinline__ int cta_swz(int r) { return ((r & 1) << 3) | ((r >> 1) & 7); }

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

constexpr int kSmemPerSm = 233472;   // shared memory of one SM (228 KB)

template <int KIND, int P_, int NT_, int RG_>
struct CtaShape {
  static constexpr int P = P_;             // padded order
  static constexpr int NT = NT_;           // threads
  static constexpr int B = 8;              // panel width
  static constexpr int TGC = 8;            // thread columns of the update tiling
  static constexpr int TGR = NT / TGC;     // thread rows
  static constexpr int CB = P / TGC;       // columns per thread (tc + 8 c)
  static constexpr int RB = P / TGR;       // rows per thread (tr + TGR r)
  static constexpr int RG = RG_;           // rows updated together
  static constexpr int RPL = (P + 31) / 32;   // panel rows per lane of warp 0
  static constexpr int MS = B + 1;         // multiplier row stride (odd)
  static constexpr int off_Mm = P * P;
  static constexpr int off_V = off_Mm + P * MS;
  static constexpr int off_r = off_V + B * P;
  static constexpr int n_dbl = off_r + B;
  static constexpr int n_int = 2 * P + 4;
  static constexpr size_t dyn_smem = size_t(n_dbl) * 8 + size_t(n_int) * 4;
  static constexpr int by_smem = int(kSmemPerSm / (dyn_smem + 1024));
  static constexpr int by_thr = 2048 / NT;
  static constexpr int min_blocks0 = by_smem < by_thr ? by_smem : by_thr;
  static constexpr int min_blocks = min_blocks0 < 1 ? 1 : min_blocks0;
  static_assert(P % 16 == 0, "swizzle works on 16-column groups");
  static_assert(NT % 32 == 0 && TGR % 4 == 0, "4 thread rows x 8 thread columns per warp");
  static_assert(P % TGR == 0 && RB % RG == 0, "whole row groups");
  static_assert(NT >= P && NT % P == 0, "one thread per column in the pivot-row phase and the copies");
  static_assert(dyn_smem <= 232448, "one CTA's shared memory");
};

template <int KIND, int P, int NT, int RG>
__global__ void __launch_bounds__(NT, (CtaShape<KIND, P, NT, RG>::min_blocks))
cta_exact_kernel(BatchView bv) {
  using Sh = CtaShape<KIND, P, NT, RG>;
  constexpr int B = Sh::B, MS = Sh::MS, CB = Sh::CB, TGR = Sh::TGR, RB = Sh::RB, RPL = Sh::RPL;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) double dsm[];
  double* M = dsm;                         // [P][P] the matrix, swizzled
  double* Mm = dsm + Sh::off_Mm;           // [P][MS] multipliers of this panel, by row
  double* Vs = dsm + Sh::off_V;            // [B][P] pivot rows at their own step
  double* rinv_s = dsm + Sh::off_r;        // [B] fl(1/u) of this panel's pivots
  int* ps_s = reinterpret_cast<int*>(dsm + Sh::n_dbl);   // [P] position of each row
  int* perm = ps_s + P;                    // [P] row at each position
  int* flags = perm + P;                   // [0] singular

  const int t = threadIdx.x;
  const int wid = t >> 5, wl = t & 31;
  const int tc = t % Sh::TGC, tr = t / Sh::TGC;

  for (int item = blockIdx.x; item < bv.count; item += gridDim.x) {
    const int s = bv.list[item];
    const int n = bv.n[s];
    const double* __restrict__ Ag = bv.A + bv.offA[s];

    // ---- load: rows < n straight into the swizzled layout, padding columns zeroed
    {
      const int col = t % P;
      for (int row = t / P; row < n; row += NT / P) {
        double* dst = M + row * P + (col ^ cta_swz(row));
        if (col < n) cp_async8(dst, Ag + int64_t(row) * n + col);
        else *dst = 0.0;
      }
      if (t < P) { ps_s[t] = t; perm[t] = t; }
      if (t == 0) flags[0] = 0;
      cp_async_wait_all();
      __syncthreads();
    }

    const int npan = (n + B - 1) / B;
    bool singular = false;
    for (int jb = 0; jb < npan; ++jb) {
      const int j0 = jb * B;
      const int nb = min(B, n - j0);

      // ---- 1. warp 0 factorises the panel in its registers -------------------
      // Lane l holds rows l, l+32, ...; the panel is kept rotated so that the
      // current pivot column is always register column 0.
      if (wid == 0) {
        double pr[RPL][B];
        int ps[RPL];
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          const int r = wl + 32 * i;
          const bool live = (RPL * 32 == P || r < P) && r < n;
          ps[i] = live ? ps_s[r] : 0x7fffffff;
          const int sw = cta_swz(r);
#pragma unroll
          for (int c = 0; c < B; ++c) pr[i][c] = live ? M[r * P + ((j0 + c) ^ sw)] : 0.0;
          if (live && nb < B) {
            // multipliers of the steps a short last panel does not take are zero
#pragma unroll
            for (int c = 0; c < B; ++c)
              if (c >= nb) Mm[r * MS + c] = 0.0;
          }
        }
        bool sing = false;
        int k = 0;
        // Software pipelining: a step updates at once only the column the next
        // pivot search reads; its other columns are updated at the start of the
        // next step, while that step's reduction is in flight.  dmode: 0 nothing
        // pending, 1 subtract dl * dpv, 2 scale by drinv (the pivot row); dpv is
        // the pending step's pivot row in that step's register frame.
        int dmode[RPL];
        double dl[RPL], dpv[B];
        double drinv = 0.0;
        int dk = 0;
#pragma unroll
        for (int i = 0; i < RPL; ++i) { dmode[i] = 0; dl[i] = 0.0; }
#pragma unroll
        for (int c = 0; c < B; ++c) dpv[c] = 0.0;
        auto apply_pending = [&]() {
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
#pragma unroll
            for (int c = 2; c < B; ++c) {
              if (dmode[i] == 1 && (KIND == kInvert || dk + c < B))
                pr[i][c - 1] = sub_rn(pr[i][c - 1], mul_rn(dl[i], dpv[c]));
              if (KIND == kInvert && dmode[i] == 2) pr[i][c - 1] = mul_rn(pr[i][c - 1], drinv);
            }
            dmode[i] = 0;
          }
        };
#pragma unroll 2
        for (; k < nb; ++k) {
          const int j = j0 + k;
          // this lane's best candidate: larger |a| first, then smaller position;
          // eligible rows carry bit 63, NaN counts as zero (cblas idamax)
          unsigned long long kb = 0ull;
          unsigned pb = 0xffffffffu;
          double vb = 1.0;
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const int r = wl + 32 * i;
            if (r < n && ps[i] >= j) {
              const double v = fabs(pr[i][0]);
              const unsigned long long key =
                  (v == v) ? (static_cast<unsigned long long>(__double_as_longlong(v)) | (1ull << 63)) : (1ull << 63);
              if (key > kb || (key == kb && unsigned(ps[i]) < pb)) { kb = key; pb = unsigned(ps[i]); vb = pr[i][0]; }
            }
          }
          // reciprocal of the lane's own candidate, overlapping the reduction
          const double rb = __drcp_rn(vb);
          const unsigned hi = unsigned(kb >> 32), lo = unsigned(kb);
          const unsigned mh = __reduce_max_sync(FULL, hi);
          const unsigned ml = __reduce_max_sync(FULL, hi == mh ? lo : 0u);
          const int ppos = int(__reduce_min_sync(FULL, (hi == mh && lo == ml) ? pb : 0xffffffffu));
          apply_pending();
          int pi = 0;
          bool own = false;
#pragma unroll
          for (int i = 0; i < RPL; ++i)
            if (ps[i] == ppos) { pi = i; own = true; }
          const int pl = __ffs(__ballot_sync(FULL, own)) - 1;
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            if (ps[i] == ppos) ps[i] = j;
            else if (ps[i] == j) ps[i] = ppos;
          }
          double pv[B];
#pragma unroll
          for (int c = 0; c < B; ++c) {
            double mine = pr[0][c];
#pragma unroll
            for (int i = 1; i < RPL; ++i) mine = (pi == i) ? pr[i][c] : mine;
            pv[c] = __shfl_sync(FULL, mine, pl);
          }
          const double rinv = __shfl_sync(FULL, rb, pl);   // = fl(1/u_jj), correctly rounded
          const double ujj = pv[0];
          if (__any_sync(FULL, ujj == 0.0)) { sing = true; break; }
          double lrow[RPL];
#pragma unroll
          for (int i = 0; i < RPL; ++i) lrow[i] = mul_rn(pr[i][0], rinv);
          if (!(fabs(ujj) >= kDblMin)) {
            // GSL divides by a pivot below DBL_MIN instead of scaling (lu.c:170-176)
#pragma unroll
            for (int i = 0; i < RPL; ++i)
              if (ps[i] > j) lrow[i] = div_rn(pr[i][0], ujj);
          }
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const int r = wl + 32 * i;
            const bool is_piv = (ps[i] == j);
            const bool below = ps[i] > j;
            const bool upd = r < n && !is_piv && (KIND == kInvert || below);
            dmode[i] = upd ? 1 : ((KIND == kInvert && is_piv) ? 2 : 0);
            dl[i] = lrow[i];
            if (upd) {
              Mm[r * MS + k] = lrow[i];
              if (KIND == kInvert || k + 1 < B) pr[i][1] = sub_rn(pr[i][1], mul_rn(lrow[i], pv[1]));
              pr[i][0] = (KIND == kInvert) ? -lrow[i] : lrow[i];
            }
            if (KIND == kInvert && is_piv) {
              pr[i][0] = rinv;
              pr[i][1] = mul_rn(pr[i][1], rinv);
            }
          }
#pragma unroll
          for (int c = 0; c < B; ++c) dpv[c] = pv[c];
          drinv = rinv;
          dk = k;
          if (wl == 0) rinv_s[k] = rinv;
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const double first = pr[i][0];
#pragma unroll
            for (int c = 0; c < B - 1; ++c) pr[i][c] = pr[i][c + 1];
            pr[i][B - 1] = first;
          }
        }
        if (!sing) apply_pending();
        if (sing) {
          if (wl == 0) flags[0] = 1;
        } else {
#pragma unroll 1
          for (; k < B; ++k) {
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
              const double first = pr[i][0];
#pragma unroll
              for (int c = 0; c < B - 1; ++c) pr[i][c] = pr[i][c + 1];
              pr[i][B - 1] = first;
            }
          }
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const int r = wl + 32 * i;
            if ((RPL * 32 == P || r < P) && r < n) {
              const int sw = cta_swz(r);
#pragma unroll
              for (int c = 0; c < B; ++c) M[r * P + ((j0 + c) ^ sw)] = pr[i][c];
              ps_s[r] = ps[i];
              perm[ps[i]] = r;
            }
          }
        }
      }
      __syncthreads();
      if (flags[0]) { singular = true; break; }

      // ---- 2. the panel's pivot rows at their own step, one thread per column
      {
        const int c = t % P;
        const bool live = (t < P) && (c < j0 || c >= j0 + B) && (KIND == kInvert || c >= j0 + B);
        if (live) {
          int q[B];
          double v[B];
#pragma unroll
          for (int k = 0; k < B; ++k) {
            q[k] = (k < nb) ? perm[j0 + k] : 0;
            v[k] = (k < nb) ? M[q[k] * P + (c ^ cta_swz(q[k]))] : 0.0;
          }
#pragma unroll
          for (int k = 1; k < B; ++k)
#pragma unroll
            for (int k2 = 0; k2 < k; ++k2)
              if (k < nb) v[k] = sub_rn(v[k], mul_rn(Mm[q[k] * MS + k2], v[k2]));
#pragma unroll
          for (int k = 0; k < B; ++k) Vs[k * P + c] = v[k];
#pragma unroll
          for (int k = 0; k < B; ++k) {
            if (k < nb) {
              double f = v[k];
              if (KIND == kInvert) {
                // scaled at its own step, then eliminated by the later pivots
                f = mul_rn(f, rinv_s[k]);
#pragma unroll
                for (int k2 = k + 1; k2 < B; ++k2)
                  if (k2 < nb) f = fma(-Mm[q[k] * MS + k2], v[k2], f);
              }
              M[q[k] * P + (c ^ cta_swz(q[k]))] = f;
            }
          }
        }
      }
      __syncthreads();

      // ---- 3. update of every other row outside the panel ----------------------
#pragma unroll 1
      for (int rg = 0; rg < RB; rg += RG) {
        int row[RG];
        bool keep[RG];
#pragma unroll
        for (int u = 0; u < RG; ++u) {
          row[u] = tr + TGR * (rg + u);
          const int p = ps_s[row[u]];
          keep[u] = row[u] < n && (p < j0 || p >= j0 + nb) && (KIND == kInvert || p >= j0 + B);
        }
        double a[RG][CB];
#pragma unroll
        for (int u = 0; u < RG; ++u) {
          const int sw = cta_swz(row[u]);
#pragma unroll
          for (int c = 0; c < CB; ++c) a[u][c] = M[row[u] * P + ((tc + 8 * c) ^ sw)];
        }
#pragma unroll
        for (int k = 0; k < B; ++k) {
          double mk[RG], vk[CB];
#pragma unroll
          for (int u = 0; u < RG; ++u) mk[u] = Mm[row[u] * MS + k];
#pragma unroll
          for (int c = 0; c < CB; ++c) vk[c] = Vs[k * P + tc + 8 * c];
#pragma unroll
          for (int u = 0; u < RG; ++u)
#pragma unroll
            for (int c = 0; c < CB; ++c) a[u][c] = sub_rn(a[u][c], mul_rn(mk[u], vk[c]));
        }
#pragma unroll
        for (int u = 0; u < RG; ++u) {
          if (keep[u]) {
            const int sw = cta_swz(row[u]);
#pragma unroll
            for (int c = 0; c < CB; ++c)
              if (c != jb && (KIND == kInvert || c > jb)) M[row[u] * P + ((tc + 8 * c) ^ sw)] = a[u][c];
          }
        }
      }
      __syncthreads();
    }

    if (singular) {
      if (t == 0) {
        bv.status[s] = (KIND == kSolve) ? kSolveSingular : kInvertSingular;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
      __syncthreads();
      continue;
    }

    if (KIND == kInvert) {
      // A^-1[q][c] = W[q][ps[c]] with W the physically permuted array, i.e.
      // row perm[q] of the in-place result (A^-1 = W P, P from GSL's permutation)
      double* __restrict__ Og = bv.out + bv.offA[s];
      const int c = t % P;
      if (c < n) {
        const int pc = ps_s[c];
        for (int q = t / P; q < n; q += NT / P) {
          const int r = perm[q];
          Og[int64_t(q) * n + c] = M[r * P + (pc ^ cta_swz(r))];
        }
      }
      if (t == 0) {
        bv.status[s] = kOk;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
    } else {
      // LU_svx (lu.c:324-360): permute b, unit-lower then upper sweep, each entry
      // in GSL's order; row q of the factors is row perm[q] of M
      double* vec = Vs;                    // [P] (Vs holds B*P >= 2P doubles)
      double* xs = Vs + P;
      if (wid == 0) {
        const int64_t ov = bv.offv[s];
        for (int i = wl; i < n; i += 32) vec[i] = bv.b[ov + perm[i]];
        __syncwarp();
        for (int j = 0; j < n; ++j) {
          const double yj = vec[j];
          for (int i = j + 1 + wl; i < n; i += 32) {
            const int r = perm[i];
            vec[i] = sub_rn(vec[i], mul_rn(M[r * P + (j ^ cta_swz(r))], yj));
          }
          __syncwarp();
        }
        if (wl == 0) {
          for (int i = n - 1; i >= 0; --i) {
            const int r = perm[i], sw = cta_swz(r);
            double u = vec[i];
            for (int k = i + 1; k < n; ++k) u = sub_rn(u, mul_rn(M[r * P + (k ^ sw)], xs[k]));
            xs[i] = div_rn(u, M[r * P + (i ^ sw)]);
          }
        }
        __syncwarp();
        // residual check on the original A (matrix_cpu.c:155-187), first failing row decides
        int first = 0x7fffffff, fcode = 0;
        for (int i = wl; i < n; i += 32) {
          double acc = 0.0;
          const double* __restrict__ arow = Ag + int64_t(i) * n;
          for (int k = 0; k < n; ++k) acc = add_rn(acc, mul_rn(arow[k], xs[k]));
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
          const int of = __shfl_xor_sync(FULL, first, off);
          const int oc = __shfl_xor_sync(FULL, fcode, off);
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
