// CTA-per-system kernels for 32 < n <= 256 (macro-atom jumping matrices of a
// few dozen to a few hundred levels, per-element macro populations).
//
// The padded P x P matrix is held row-major with its columns XOR-swizzled
// inside 16-column groups (row, column and tile accesses are then free of
// shared-memory bank conflicts and stay inside one 128-byte line): in shared
// memory for the smallest classes, in an L2-resident global workspace slab per
// CTA above them, where several CTAs per SM keep several pivot chains in flight.  Rows
// never move: each physical row carries its current position (ps), and
// perm[q] names the row at position q, so GSL's row swaps cost two integer
// stores and ties in the pivot search break on positions exactly as GSL's
// physical swaps would.  The factorisation is blocked by panels of B = 8
// columns.  Per panel:
//   1. the panel warps factorise the n x B panel in registers (GSL's
//      LU_decomp_L2 on a panel, lu.c:129-191): first strict maximum pivot by a
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

// barrier 1 over the first `count` threads (the panel warps)
__device__ __forceinline__ void panel_bar(int count) { asm volatile("bar.sync 1, %0;\n" ::"r"(count) : "memory"); }

constexpr int kSmemPerSm = 233472;   // shared memory of one SM (228 KB)

// P: padded order; NT: threads; RG x CC: rows x columns of one update tile of
// the workspace classes (columns tc + 8c; the shared-memory classes update one
// column at a time); PW: panel warps; GM: matrix in a global workspace slab;
// MINB: CTAs per SM asked of the register allocator (0: as many as fit).
template <int KIND, int P_, int NT_, int RG_, int CC_, int PW_, bool GM_, int MINB_>
struct CtaShape {
  static constexpr int P = P_;
  static constexpr int NT = NT_;
  static constexpr int NW = NT / 32;
  static constexpr int B = 8;              // panel width
  static constexpr int TGC = 8;            // thread columns of the update tiling
  static constexpr int TGR = NT / TGC;     // thread rows
  static constexpr int CB = P / TGC;       // columns per thread (tc + 8 c)
  static constexpr int RB = P / TGR;       // rows per thread (tr + TGR r)
  static constexpr int RG = RG_;
  static constexpr int CC = CC_;
  static constexpr int PW = PW_;
  static constexpr int PT = 32 * PW;       // panel threads
  static constexpr int RPL = (P + PT - 1) / PT;   // panel rows per panel thread
  static constexpr bool GM = GM_;
  static constexpr int MS = B + 1;         // multiplier row stride (odd)
  static constexpr int off_Mm = GM ? 0 : P * P;
  static constexpr int off_V = off_Mm + P * MS;
  static constexpr int off_r = off_V + B * P;
  static constexpr int off_pb = off_r + B; // pivot-row exchange of a multi-warp panel
  static constexpr int n_dbl = off_pb + B + 2;
  static constexpr int n_int = 2 * P + 4 + 4 * PW;
  static constexpr size_t dyn_smem = size_t(n_dbl) * 8 + size_t(n_int) * 4;
  static constexpr int by_smem = int(kSmemPerSm / (dyn_smem + 1024));
  static constexpr int by_thr = 2048 / NT;
  static constexpr int min_blocks0 = by_smem < by_thr ? by_smem : by_thr;
  static constexpr int min_blocks1 = (MINB_ > 0 && MINB_ < min_blocks0) ? MINB_ : min_blocks0;
  static constexpr int min_blocks = min_blocks1 < 1 ? 1 : min_blocks1;
  static constexpr int64_t slab = GM ? int64_t(P) * P : 0;   // workspace doubles per CTA
  static_assert(P % 16 == 0, "swizzle works on 16-column groups");
  static_assert(NT % 32 == 0 && TGR % 4 == 0, "4 thread rows x 8 thread columns per warp");
  static_assert(P % TGR == 0 && RB % RG == 0 && CB % CC == 0, "whole update tiles");
  static_assert(PW >= 1 && PW <= NW, "panel warps are warps of the CTA");
  static_assert(dyn_smem <= 232448, "one CTA's shared memory");
};

template <int KIND, int P, int NT, int RG, int CC, int PW, bool GM, int MINB>
__global__ void __launch_bounds__(NT, (CtaShape<KIND, P, NT, RG, CC, PW, GM, MINB>::min_blocks))
cta_exact_kernel(BatchView bv, double* __restrict__ work) {
  using Sh = CtaShape<KIND, P, NT, RG, CC, PW, GM, MINB>;
  constexpr int B = Sh::B, MS = Sh::MS, CB = Sh::CB, TGR = Sh::TGR, RB = Sh::RB, RPL = Sh::RPL;
  constexpr int PT = Sh::PT, NW = Sh::NW;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) double dsm[];
  double* M = GM ? work + int64_t(blockIdx.x) * Sh::slab : dsm;   // [P][P] the matrix, swizzled
  double* Mm = dsm + Sh::off_Mm;           // [P][MS] multipliers of this panel, by row
  double* Vs = dsm + Sh::off_V;            // [B][P] pivot rows at their own step
  double* rinv_s = dsm + Sh::off_r;        // [B] fl(1/u) of this panel's pivots
  double* pivbuf = dsm + Sh::off_pb;       // [B+1] pivot row and its reciprocal (PW > 1)
  int* ps_s = reinterpret_cast<int*>(dsm + Sh::n_dbl);   // [P] position of each row
  int* perm = ps_s + P;                    // [P] row at each position
  int* flags = perm + P;                   // [0] singular, [1] an infinite pivot
  unsigned* cand = reinterpret_cast<unsigned*>(flags + 4);   // [PW][4] per-warp pivot candidates

  const int t = threadIdx.x;
  const int wid = t >> 5, wl = t & 31;
  const int tc = t % Sh::TGC, tr = t / Sh::TGC;

  const int count = batch_count(bv);
  for (int item = blockIdx.x; item < count; item += gridDim.x) {
    const int s = bv.list[item];
    const int n = bv.n[s];
    const double* __restrict__ Ag = bv.A + bv.offA[s];

    // ---- load: rows < n into the swizzled layout, padding columns zeroed; a
    // warp per row, consecutive lanes on consecutive columns
    for (int row = wid; row < n; row += NW) {
      const int sw = cta_swz(row);
      const double* __restrict__ src = Ag + int64_t(row) * n;
#pragma unroll 4
      for (int col = wl; col < P; col += 32) {
        double* dst = M + row * P + (col ^ sw);
        if (GM) *dst = (col < n) ? __ldg(src + col) : 0.0;
        else if (col < n) cp_async8(dst, src + col);
        else *dst = 0.0;
      }
    }
    for (int r = t; r < P; r += NT) { ps_s[r] = r; perm[r] = r; }
    if (t == 0) {
      flags[0] = 0;
      flags[1] = 0;
    }
    if (!GM) cp_async_wait_all();
    __syncthreads();

    const int npan = (n + B - 1) / B;
    bool singular = false;
    for (int jb = 0; jb < npan; ++jb) {
      const int j0 = jb * B;
      const int nb = min(B, n - j0);

      // ---- 1. the panel warps factorise the panel in their registers ----------
      // Panel thread p holds rows p, p + PT, ...; the panel is kept rotated so
      // that the current pivot column is always register column 0.
      if (wid < PW) {
        double pr[RPL][B];
        int ps[RPL];
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          const int r = t + PT * i;
          const bool live = (RPL * PT == P || r < P) && r < n;
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
        // the pending step's pivot row in that step's register frame.  The
        // pivot row's registers hold dpv itself, so its scaled values are the
        // same for every lane, and each row takes its new value by selection:
        // no lane-dependent branches in the panel.
        int dmode[RPL];
        double dl[RPL], dpv[B];
        double drinv = 0.0;
        int dk = 0;
#pragma unroll
        for (int i = 0; i < RPL; ++i) { dmode[i] = 0; dl[i] = 0.0; }
#pragma unroll
        for (int c = 0; c < B; ++c) dpv[c] = 0.0;
        auto apply_pending = [&]() {
          double sv[B];
#pragma unroll
          for (int c = 2; c < B; ++c) sv[c] = (KIND == kInvert) ? mul_rn(dpv[c], drinv) : 0.0;
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
#pragma unroll
            for (int c = 2; c < B; ++c) {
              const double x = sub_rn(pr[i][c - 1], mul_rn(dl[i], dpv[c]));
              if (KIND == kInvert) pr[i][c - 1] = dmode[i] == 2 ? sv[c] : (dmode[i] == 1 ? x : pr[i][c - 1]);
              else pr[i][c - 1] = (dmode[i] == 1 && dk + c < B) ? x : pr[i][c - 1];
            }
            dmode[i] = 0;
          }
        };
#pragma unroll 2
        for (; k < nb; ++k) {
          const int j = j0 + k;
          // this thread's best candidate: larger |a| first, then smaller position;
          // eligible rows carry bit 63, NaN counts as zero (cblas idamax)
          unsigned long long kb = 0ull;
          unsigned pb = 0xffffffffu;
          double vb = 1.0;
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const int r = t + PT * i;
            if (r < n && ps[i] >= j) {
              const double v = fabs(pr[i][0]);
              const unsigned long long key =
                  (v == v) ? (static_cast<unsigned long long>(__double_as_longlong(v)) | (1ull << 63)) : (1ull << 63);
              if (key > kb || (key == kb && unsigned(ps[i]) < pb)) { kb = key; pb = unsigned(ps[i]); vb = pr[i][0]; }
            }
          }
          // reciprocal of the thread's own candidate, overlapping the reduction
          const double rb = __drcp_rn(vb);
          const unsigned hi = unsigned(kb >> 32), lo = unsigned(kb);
          const unsigned mh = __reduce_max_sync(FULL, hi);
          const unsigned ml = __reduce_max_sync(FULL, hi == mh ? lo : 0u);
          int ppos = int(__reduce_min_sync(FULL, (hi == mh && lo == ml) ? pb : 0xffffffffu));
          if (PW > 1) {
            // best of the panel warps' candidates, same order
            if (wl == 0) { cand[4 * wid] = mh; cand[4 * wid + 1] = ml; cand[4 * wid + 2] = unsigned(ppos); }
            panel_bar(PT);
            unsigned bh = cand[0], bl = cand[1], bp = cand[2];
#pragma unroll
            for (int w = 1; w < PW; ++w) {
              const unsigned h2 = cand[4 * w], l2 = cand[4 * w + 1], p2 = cand[4 * w + 2];
              if (h2 > bh || (h2 == bh && (l2 > bl || (l2 == bl && p2 < bp)))) { bh = h2; bl = l2; bp = p2; }
            }
            ppos = int(bp);
          }
          apply_pending();
          int pi = 0;
          bool own = false;
#pragma unroll
          for (int i = 0; i < RPL; ++i)
            if (ps[i] == ppos) { pi = i; own = true; }
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            if (ps[i] == ppos) ps[i] = j;
            else if (ps[i] == j) ps[i] = ppos;
          }
          double pv[B];
          double rinv;
          if (PW > 1) {
            if (own) {
#pragma unroll
              for (int c = 0; c < B; ++c) {
                double mine = pr[0][c];
#pragma unroll
                for (int i = 1; i < RPL; ++i) mine = (pi == i) ? pr[i][c] : mine;
                pivbuf[c] = mine;
              }
              pivbuf[B] = rb;
            }
            panel_bar(PT);
#pragma unroll
            for (int c = 0; c < B; ++c) pv[c] = pivbuf[c];
            rinv = pivbuf[B];
          } else {
            const int pl = __ffs(__ballot_sync(FULL, own)) - 1;
#pragma unroll
            for (int c = 0; c < B; ++c) {
              double mine = pr[0][c];
#pragma unroll
              for (int i = 1; i < RPL; ++i) mine = (pi == i) ? pr[i][c] : mine;
              pv[c] = __shfl_sync(FULL, mine, pl);
            }
            rinv = __shfl_sync(FULL, rb, pl);   // = fl(1/u_jj), correctly rounded
          }
          const double ujj = pv[0];
          if (__any_sync(FULL, ujj == 0.0)) { sing = true; break; }
          if (KIND == kInvert && t == 0 && isinf(ujj)) flags[1] = 1;
          double lrow[RPL];
#pragma unroll
          for (int i = 0; i < RPL; ++i) lrow[i] = mul_rn(pr[i][0], rinv);
          if (!(fabs(ujj) >= kDblMin)) {
            // GSL divides by a pivot below DBL_MIN instead of scaling (lu.c:170-176)
#pragma unroll
            for (int i = 0; i < RPL; ++i)
              if (ps[i] > j) lrow[i] = div_rn(pr[i][0], ujj);
          }
          const double s1 = (KIND == kInvert) ? mul_rn(pv[1], rinv) : 0.0;
#pragma unroll
          for (int i = 0; i < RPL; ++i) {
            const int r = t + PT * i;
            const bool is_piv = (ps[i] == j);
            const bool below = ps[i] > j;
            const bool upd = r < n && !is_piv && (KIND == kInvert || below);
            dmode[i] = upd ? 1 : ((KIND == kInvert && is_piv) ? 2 : 0);
            dl[i] = lrow[i];
            if (upd) Mm[r * MS + k] = lrow[i];
            const double x1 = sub_rn(pr[i][1], mul_rn(lrow[i], pv[1]));
            if (KIND == kInvert) {
              // the pivot row holds pv: its scaled entry is s1 on every lane
              pr[i][1] = upd ? x1 : (is_piv ? s1 : pr[i][1]);
              pr[i][0] = upd ? -lrow[i] : (is_piv ? rinv : pr[i][0]);
            } else {
              if (k + 1 < B) pr[i][1] = upd ? x1 : pr[i][1];
              pr[i][0] = upd ? lrow[i] : pr[i][0];
            }
          }
#pragma unroll
          for (int c = 0; c < B; ++c) dpv[c] = pv[c];
          drinv = rinv;
          dk = k;
          if (t == 0) rinv_s[k] = rinv;
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
          if (t == 0) flags[0] = 1;
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
            const int r = t + PT * i;
            if ((RPL * PT == P || r < P) && r < n) {
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
      for (int c = t; c < P; c += NT) {
        if (!((c < j0 || c >= j0 + B) && (KIND == kInvert || c >= j0 + B))) continue;
        if constexpr (!GM) {
          // Every load is issued before the dependent chains: positions j0 + k < P
          // hold a valid row even past a short last panel (rows >= n keep their
          // own position), so the loads need no guard and the steps that panel
          // does not take only select zeros.
          int q[B];
          double v[B];
#pragma unroll
          for (int k = 0; k < B; ++k) q[k] = perm[j0 + k];
#pragma unroll
          for (int k = 0; k < B; ++k) {
            const double w = M[q[k] * P + (c ^ cta_swz(q[k]))];
            v[k] = (k < nb) ? w : 0.0;
          }
#pragma unroll
          for (int k = 1; k < B; ++k) {
            double ml[B];
#pragma unroll
            for (int k2 = 0; k2 < k; ++k2) ml[k2] = Mm[q[k] * MS + k2];
#pragma unroll
            for (int k2 = 0; k2 < k; ++k2)
              if (k < nb) v[k] = sub_rn(v[k], mul_rn(ml[k2], v[k2]));
          }
          double f[B];
          if (KIND == kInvert) {
            // scaled at its own step, then eliminated by the later pivots
#pragma unroll
            for (int k = 0; k < B; ++k) {
              double mu[B];
#pragma unroll
              for (int k2 = k + 1; k2 < B; ++k2) mu[k2] = Mm[q[k] * MS + k2];
              f[k] = mul_rn(v[k], rinv_s[k]);
#pragma unroll
              for (int k2 = k + 1; k2 < B; ++k2)
                if (k2 < nb) f[k] = fma(-mu[k2], v[k2], f[k]);
            }
          } else {
#pragma unroll
            for (int k = 0; k < B; ++k) f[k] = v[k];
          }
#pragma unroll
          for (int k = 0; k < B; ++k) Vs[k * P + c] = v[k];
#pragma unroll
          for (int k = 0; k < B; ++k)
            if (k < nb) M[q[k] * P + (c ^ cta_swz(q[k]))] = f[k];
        } else {
          // the workspace classes load from L2 on demand: fewer registers
          // held across the chains, which their occupancy needs more
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
      if (!GM) {
        // Shared memory: column by column.  The panel's own columns are
        // skipped, a solve skips its L columns too, and the inverse's columns
        // left of the panel (the Gauss-Jordan inverse, never part of GSL's LU)
        // take fused updates; every other entry gets GSL's unfused
        // multiply-subtract with k ascending.
#pragma unroll 1
        for (int rg = 0; rg < RB; rg += RG) {
          int row[RG], sw[RG];
          bool keep[RG];
          double mk[B][RG];
#pragma unroll
          for (int u = 0; u < RG; ++u) {
            row[u] = tr + TGR * (rg + u);
            sw[u] = cta_swz(row[u]);
            const int p = ps_s[row[u]];
            keep[u] = row[u] < n && (p < j0 || p >= j0 + nb) && (KIND == kInvert || p >= j0 + B);
#pragma unroll
            for (int k = 0; k < B; ++k) mk[k][u] = Mm[row[u] * MS + k];
          }
#pragma unroll 2
          for (int c = 0; c < CB; ++c) {
            if (c == jb || (KIND == kSolve && c < jb)) continue;
            const int col = tc + 8 * c;
            double vk[B], a[RG];
#pragma unroll
            for (int k = 0; k < B; ++k) vk[k] = Vs[k * P + col];
#pragma unroll
            for (int u = 0; u < RG; ++u) a[u] = M[row[u] * P + (col ^ sw[u])];
            if (KIND == kInvert && c < jb) {
#pragma unroll
              for (int k = 0; k < B; ++k)
#pragma unroll
                for (int u = 0; u < RG; ++u) a[u] = fma(-mk[k][u], vk[k], a[u]);
            } else {
#pragma unroll
              for (int k = 0; k < B; ++k)
#pragma unroll
                for (int u = 0; u < RG; ++u) a[u] = sub_rn(a[u], mul_rn(mk[k][u], vk[k]));
            }
#pragma unroll
            for (int u = 0; u < RG; ++u)
              if (keep[u]) M[row[u] * P + (col ^ sw[u])] = a[u];
          }
        }
      } else {
        // Global workspace: RG x CC tiles, every load of a tile in flight
        // together to cover the L2 latency; GSL's unfused multiply-subtract
        // with k ascending except on tiles wholly left of the panel.
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
#pragma unroll 1
          for (int cg = 0; cg < CB; cg += CC) {
            // a chunk wholly left of the panel: fused updates for an inverse
            // (outside GSL's LU), nothing to do for a solve (its L columns).
            // The rule is per chunk, so the candidates of one order share CC.
            const bool left = cg + CC <= jb;
            if (KIND == kSolve && left) continue;
            double a[RG][CC];
#pragma unroll
            for (int u = 0; u < RG; ++u) {
              const int sw = cta_swz(row[u]);
#pragma unroll
              for (int c = 0; c < CC; ++c) a[u][c] = M[row[u] * P + ((tc + 8 * (cg + c)) ^ sw)];
            }
            if (left) {
#pragma unroll
              for (int k = 0; k < B; ++k) {
                double mk[RG], vk[CC];
#pragma unroll
                for (int u = 0; u < RG; ++u) mk[u] = Mm[row[u] * MS + k];
#pragma unroll
                for (int c = 0; c < CC; ++c) vk[c] = Vs[k * P + tc + 8 * (cg + c)];
#pragma unroll
                for (int u = 0; u < RG; ++u)
#pragma unroll
                  for (int c = 0; c < CC; ++c) a[u][c] = fma(-mk[u], vk[c], a[u][c]);
              }
            } else {
#pragma unroll
              for (int k = 0; k < B; ++k) {
                double mk[RG], vk[CC];
#pragma unroll
                for (int u = 0; u < RG; ++u) mk[u] = Mm[row[u] * MS + k];
#pragma unroll
                for (int c = 0; c < CC; ++c) vk[c] = Vs[k * P + tc + 8 * (cg + c)];
#pragma unroll
                for (int u = 0; u < RG; ++u)
#pragma unroll
                  for (int c = 0; c < CC; ++c) a[u][c] = sub_rn(a[u][c], mul_rn(mk[u], vk[c]));
              }
            }
#pragma unroll
            for (int u = 0; u < RG; ++u) {
              if (keep[u]) {
                const int sw = cta_swz(row[u]);
#pragma unroll
                for (int c = 0; c < CC; ++c) {
                  const int cb = cg + c;
                  if (cb != jb && (KIND == kInvert || cb > jb)) M[row[u] * P + ((tc + 8 * cb) ^ sw)] = a[u][c];
                }
              }
            }
          }
        }
      }
      __syncthreads();
    }

    if (singular || (KIND == kInvert && flags[1])) {
      // a zero pivot: GSL_EDOM; for an inverse, an infinite one: GSL_ESING
      // (LU_invx finds 1/u_jj = 0 after inverting U); the output is untouched
      if (t == 0) {
        bv.status[s] = (KIND == kSolve) ? kSolveSingular : (singular ? kInvertSingular : kInvertInfPivot);
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
      __syncthreads();
      continue;
    }

    if (KIND == kInvert) {
      // A^-1[q][c] = W[q][ps[c]] with W the physically permuted array, i.e.
      // row perm[q] of the in-place result (A^-1 = W P, P from GSL's permutation);
      // a warp per output row
      double* __restrict__ Og = bv.out + bv.offA[s];
      for (int q = wid; q < n; q += NW) {
        const int r = perm[q], sw = cta_swz(r);
        double* __restrict__ orow = Og + int64_t(q) * n;
        for (int c = wl; c < n; c += 32) orow[c] = M[r * P + (ps_s[c] ^ sw)];
      }
      if (t == 0) {
        bv.status[s] = kOk;
        if (bv.diag) bv.diag[s] = kDiagExact;
      }
    } else {
      // LU_svx (lu.c:324-360): permute b, unit-lower then upper sweep, each entry
      // in GSL's order; row q of the factors is row perm[q] of M
      double* vec = Vs;                    // [P]
      double* xs = Vs + P;                 // [P]
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
