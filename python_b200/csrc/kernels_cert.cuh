// Certified inverse: Gauss-Jordan without pivoting for nonsingular M-matrices.
//
// The macro-atom jumping matrix N = I - Q / Q_norm that calc_matom_matrix
// inverts (reference source/macro_accelerate.c:268-284, inverted at :315) has a
// unit diagonal, non-positive off-diagonal entries and off-diagonal row sums
// 1 - R / Q_norm < 1 wherever the level can deactivate: a Z-matrix that is
// strictly diagonally dominant by rows, i.e. a nonsingular M-matrix.  For such
// a matrix
//   * Gaussian elimination needs no pivoting: every Schur complement stays a
//     row-dominant M-matrix, the growth factor is at most 2, and an
//     off-diagonal update subtracts a product of two non-positive numbers from
//     a non-positive one (no cancellation);
//   * no exact-zero pivot can occur in GSL's partial-pivoting LU either, so the
//     reference returns code 0 (lu.c:540 `singular` never fires) and the only
//     question is accuracy.
// The certificate checked per matrix, on the FP64 input, is
//     a_rr > 0,  a_rc <= 0 (c != r),  sum_{c != r} |a_rc| * (1 + 2^-40) <= (1 - tau) a_rr
// for every row r, tau = kCertMargin, with every entry finite.  Measured against
// the reference's GSL inverse on M-matrices whose every row sits at the margin,
// the no-pivot result differs by <= 4e-12 (relative, max-abs) at tau = 1e-5 and
// grows like 1/tau below it; macro-atom matrices with realistic deactivation
// probabilities (>= 1e-4) stay below 2e-15.  A matrix that fails the
// certificate (a level that cannot deactivate, any positive off-diagonal
// entry, NaN / Inf) is appended to a fallback list that the GSL-exact kernels
// serve, so its result and code are the reference's.
//
// Algorithm: blocked in-place Gauss-Jordan in its rank-8 update form.  For the
// pivot block K = [kb, kb + 8), with D = W[K][K], row panel R = W[K][:] and
// column panel C = W[:][K] (old values):
//     R' = D^-1 R on columns outside K,  R' = I + D^-1 on the columns of K,
//     C' = C, minus I on the rows of K,
//     W <- W - C' R'  on every entry.
// Outside K this is the Gauss-Jordan update W - C D^-1 R; on the rows of K it
// yields D^-1 R, on the columns of K -C D^-1, and on D itself D^-1, so every
// entry takes the same fused update and no thread branches on where it sits.
//
// Layout: the padded P x P matrix is RESIDENT IN REGISTERS for the whole
// factorisation, spread over the tile threads of one CTA or of a cluster of CL
// CTAs (one SM each).  Rows go to the cluster's CTAs in blocks of 8 (block b to
// CTA b % CL); inside a CTA, tile thread (tr, tc) of an RT x CT grid holds
// local rows tr + RT i and columns tc + CT j.  Each CTA also runs one pivot
// warp that holds no tile.  Every block step moves only the two panels
// through shared memory:
//   S1  the holders of K's rows write R (transposed, RowPT[c][q]); in a
//       cluster the owner CTA's tile threads then copy that panel into every
//       other CTA, 16 bytes per store; the holders of K's columns
//       write C' (ColP[r][q], minus I on D's diagonal) locally; the holders of
//       the next pivot block write its current values (Dnext);  cluster barrier
//   S3  the tile threads form R' (RowNT[c][q]) from D^-1;     barrier
//   S4  every tile thread updates its tile, W -= C' R', while the pivot warp of
//       the CTA that owns the next block brings Dnext up to date with the same
//       fused multiply-adds, in the same order, and inverts it (8 x 8, two
//       entries per lane, shuffles), writing D^-1 of the next step into every
//       CTA of the cluster.
// So the serial 8 x 8 inverse overlaps the bulk update, and a step costs two
// barriers.
// Staging: the rows a CTA holds arrive in shared memory by 1-D TMA bulk copies
// (cp.async.bulk, one per 8-row block, completing on an mbarrier), issued for
// the NEXT matrix as soon as the current one has moved into registers, so the
// HBM latency of a matrix overlaps the factorisation of the one before.  A bulk
// copy needs 16-byte aligned ends: the aligned interior of each block is
// copied, and the at most two 8-byte ends are read by plain loads, so nothing
// outside the caller's matrix is touched.  Panel rows are 8 values at an odd stride of SP = 9 doubles, so the
// 8-byte loads of S3 and S4 -- at most 32 distinct panel rows per warp, the
// rest broadcasts -- hit distinct banks; panel buffers are double-buffered.
#pragma once
#include <cooperative_groups.h>

#include "ss_common.cuh"

namespace ss {

constexpr double kCertMargin = 1.0e-5;   // relative row-dominance margin of the certificate

// Fallback lists of the certified launches: systems that fail the certificate
// are appended, per exact-path size class, for the GSL-exact kernels.
struct CertArgs {
  const int* xcls;     // [nsys] exact-path class list of each system
  const int* fb_off;   // [classes] start of each class's list in fb_list
  int* fb_list;        // the lists
  int* fb_count;       // [classes] entries appended (zeroed before the launch)
};

// P: padded order; RT x CT: tile-thread grid of one CTA; CL: CTAs per matrix
// (a cluster); MINB: CTAs per SM asked of the register allocator.
template <int P_, int RT_, int CT_, int CL_, int MINB_>
struct CgjShape {
  static constexpr int P = P_, RT = RT_, CT = CT_, CL = CL_;
  static constexpr int NT = RT * CT;       // tile threads
  static constexpr int NTH = NT + 32;      // with the pivot warp
  static constexpr int LP = P / CL;        // rows held by one CTA
  static constexpr int TR = LP / RT;       // rows per tile thread
  static constexpr int TC = P / CT;        // columns per tile thread
  static constexpr int RB = RT / 8;        // 8-row blocks spanned by the thread rows
  static constexpr int CB = CT / 8;
  static constexpr int MINB = MINB_;
  static constexpr int SP = 9;             // stride of a panel row (8 values)
  // shared memory, in doubles, per panel buffer
  static constexpr int off_RowPT = 0;                   // [P][SP]
  static constexpr int off_RowNT = SP * P;              // [P][SP]
  static constexpr int off_ColP = 2 * SP * P;           // [LP][SP]
  static constexpr int off_Dinv = 2 * SP * P + SP * LP; // [8][SP]
  static constexpr int off_Dnext = off_Dinv + 8 * SP;   // [8][SP]
  static constexpr int buf = off_Dnext + 8 * SP;
  static constexpr int off_dg = 2 * buf;                // [LP] diagonal of each local row
  static constexpr int off_ok = off_dg + LP;            // [2][8] certificate of each CTA, by item parity
  static constexpr int off_bar = off_ok + 16;           // the staging mbarrier (8 bytes)
  static constexpr int SLOT = 8 * P + 2;                // doubles per staged 8-row block (+ alignment shift)
  static constexpr int off_stage = off_bar + 2;         // [LP / 8][SLOT], 16-byte aligned
  static constexpr int n_dbl = off_stage + (LP / 8) * SLOT;
  static constexpr size_t dyn_smem = size_t(n_dbl) * 8;
  static_assert(RT % 8 == 0 && CT % 8 == 0, "8-row / 8-column pivot blocks map onto whole thread groups");
  static_assert(CT <= 32, "a thread row's partial sums fit the reduction buffer");
  static_assert(P % (8 * CL) == 0 && LP % RT == 0 && P % CT == 0, "whole tiles");
  static_assert(NT % 32 == 0 && NTH <= 1024, "whole warps");
  static_assert(CT * LP <= 2 * buf, "certificate partials fit the panel buffers");
  static_assert((SP * P) % 2 == 0 && off_RowPT % 2 == 0, "16-byte copies of the row panel");
  static_assert(CL >= 1 && CL <= 8, "portable cluster sizes");
  static_assert(off_stage % 2 == 0 && SLOT % 2 == 0, "16-byte aligned staging slots");
  static_assert(LP / 8 <= 32, "one lane of the pivot warp issues each block's copy");
  static_assert(dyn_smem <= 232448, "one CTA's shared memory");
};

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// A barrier over every thread of the cluster: shared-memory writes made before
// it, local or into another CTA's shared memory, are visible after it.
template <int CL>
__device__ __forceinline__ void cluster_barrier() {
  if (CL > 1) cooperative_groups::this_cluster().sync();
  else __syncthreads();
}

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// one 1-D bulk copy global -> this CTA's shared memory, completing on bar
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Waits for phase `parity` of bar to complete, polling at most `limit` times;
// returns false if it never did.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit) {
  for (int it = 0; it < limit; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}
// polls of a staging wait: about a second, far beyond any copy's duration
constexpr int kStageWaitPolls = 1 << 24;

// In-place Gauss-Jordan inverse of the 8 x 8 pivot block by one warp, without
// pivoting.  Lane l holds D[l/4][2(l%4)] in d0 and D[l/4][2(l%4)+1] in d1.
// (Measured alone on an SM: ~910 cycles per call; a variant taking two pivots
// at a time through 2 x 2 determinants needed more shuffles and took ~1250.)
__device__ __forceinline__ void warp_inv8(double& d0, double& d1, int lane) {
  const int q = lane >> 2, h = lane & 3;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int kh = k >> 1;
    const double colv = (k & 1) ? d1 : d0;                 // column k lives in quarter kh
    const double dkk = __shfl_sync(0xffffffffu, colv, 4 * k + kh);
    const double f = __shfl_sync(0xffffffffu, colv, 4 * q + kh);   // D[q][k]
    const double rk0 = __shfl_sync(0xffffffffu, d0, 4 * k + h);    // D[k][2h]
    const double rk1 = __shfl_sync(0xffffffffu, d1, 4 * k + h);    // D[k][2h+1]
    const double piv = __drcp_rn(dkk);
    const double nk0 = (2 * h == k) ? piv : rk0 * piv;
    const double nk1 = (2 * h + 1 == k) ? piv : rk1 * piv;
    if (q == k) {
      d0 = nk0;
      d1 = nk1;
    } else {
      d0 = fma(-f, nk0, (2 * h == k) ? 0.0 : d0);
      d1 = fma(-f, nk1, (2 * h + 1 == k) ? 0.0 : d1);
    }
  }
}

template <int P, int RT, int CT, int CL, int MINB>
__global__ void __launch_bounds__(RT* CT + 32, MINB)
cgj_inverse_kernel(BatchView bv, CertArgs ca) {
  using S = CgjShape<P, RT, CT, CL, MINB>;
  constexpr int NT = S::NT, TR = S::TR, TC = S::TC, LP = S::LP, RB = S::RB, CB = S::CB, SP = S::SP;
  constexpr int NBLK = P / 8;
  extern __shared__ __align__(16) double sm[];
  namespace cg = cooperative_groups;

  const int tid = threadIdx.x;
  const bool tile = tid < NT;                 // warp-uniform: NT is a multiple of 32
  const int tr = tid / CT, tc = tid % CT;     // meaningful for tile threads
  const int lane = tid & 31;
  const int rank = (CL > 1) ? int(cluster_rank()) : 0;
  const int cid = blockIdx.x / CL, ncl = gridDim.x / CL;
  const int cnt = batch_count(bv);

  // global row of this thread's local row i (blocks of 8 rows dealt to the CTAs)
  auto grow = [&](int i) -> int {
    const int lr = tr + RT * i;
    return (((lr >> 3) * CL) + rank) * 8 + (lr & 7);
  };
  auto bufp = [&](int kblk) -> double* { return sm + (kblk & 1) * S::buf; };
  double W[TR][TC];

  // S1 of block kblk: the old row panel (to every CTA), the old column panel
  // minus I on D's diagonal, and the current values of the next pivot block
  auto publish = [&](int kblk) {
    double* B = bufp(kblk);
    double* RowPT = B + S::off_RowPT;
    double* ColP = B + S::off_ColP;
    const int kb = 8 * kblk;
    const int owner = kblk % CL, lbK = kblk / CL;
    if (rank == owner && (tr >> 3) == lbK % RB) {
      const int iK = lbK / RB, q = tr & 7;
      double rowv[TC];
#pragma unroll
      for (int j = 0; j < TC; ++j) rowv[j] = W[0][j];
#pragma unroll
      for (int i = 1; i < TR; ++i)
        if (i == iK) {
#pragma unroll
          for (int j = 0; j < TC; ++j) rowv[j] = W[i][j];
        }
#pragma unroll
      for (int j = 0; j < TC; ++j) RowPT[(tc + CT * j) * SP + q] = rowv[j];
    }
    if ((tc >> 3) == kblk % CB) {
      const int jK = kblk / CB, q = tc & 7;
      double colv[TR];
#pragma unroll
      for (int i = 0; i < TR; ++i) colv[i] = W[i][0];
#pragma unroll
      for (int j = 1; j < TC; ++j)
        if (j == jK) {
#pragma unroll
          for (int i = 0; i < TR; ++i) colv[i] = W[i][j];
        }
#pragma unroll
      for (int i = 0; i < TR; ++i) ColP[(tr + RT * i) * SP + q] = colv[i] - ((grow(i) == kb + q) ? 1.0 : 0.0);
    }
    if (kblk + 1 < NBLK) {
      const int k1 = kblk + 1, lbK1 = k1 / CL;
      if (rank == k1 % CL && (tr >> 3) == lbK1 % RB && (tc >> 3) == k1 % CB) {
        const int iK1 = lbK1 / RB, jK1 = k1 / CB;
        double v = W[0][0];
#pragma unroll
        for (int i = 0; i < TR; ++i)
#pragma unroll
          for (int j = 0; j < TC; ++j)
            if (i == iK1 && j == jK1) v = W[i][j];
        B[S::off_Dnext + (tr & 7) * SP + (tc & 7)] = v;
      }
    }
  };

  // cluster: the owner of block kblk copies its row panel into every other
  // CTA once its tile threads have written it (a barrier over the tile threads
  // only, so the pivot warp's work is not waited for), 16 bytes per store,
  // consecutive threads on consecutive addresses
  auto share_row_panel = [&](int kblk) {
    if (CL > 1) {
      asm volatile("bar.sync 1, %0;\n" ::"r"(NT) : "memory");
      if (rank == kblk % CL) {
        cg::cluster_group cl = cg::this_cluster();
        const double2* src = reinterpret_cast<const double2*>(bufp(kblk) + S::off_RowPT);
        for (int pr = 0; pr < CL; ++pr) {
          if (pr == rank) continue;
          double2* dst = reinterpret_cast<double2*>(cl.map_shared_rank(bufp(kblk) + S::off_RowPT, pr));
          for (int e = tid; e < P * SP / 2; e += NT) dst[e] = src[e];
        }
      }
    }
  };

  // the pivot warp: D^-1 of block kblk from the 8 x 8 values d0, d1 (lane
  // layout of warp_inv8), written into every CTA's buffer of that block
  auto pivot_inverse = [&](int kblk, double d0, double d1) {
    warp_inv8(d0, d1, lane);
    double* Dinv = bufp(kblk) + S::off_Dinv;
    const int q = lane >> 2, h = lane & 3;
    Dinv[q * SP + 2 * h] = d0;
    Dinv[q * SP + 2 * h + 1] = d1;
    if (CL > 1) {
      cg::cluster_group cl = cg::this_cluster();
#pragma unroll
      for (int pr = 0; pr < CL; ++pr) {
        if (pr == rank) continue;
        double* rp = cl.map_shared_rank(Dinv, pr);
        rp[q * SP + 2 * h] = d0;
        rp[q * SP + 2 * h + 1] = d1;
      }
    }
  };

  // ---- staging of the rows this CTA holds (pivot warp): one bulk copy of the
  // 16-byte aligned interior of each 8-row block; element e of block lb sits
  // at slot index lb * SLOT + shift + e, shift = 1 when the block starts 8
  // bytes past a 16-byte boundary
  double* stage = sm + S::off_stage;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + S::off_bar);
  auto block_span = [&](int s2, int lb, uintptr_t& b0, uintptr_t& b1) -> bool {
    const int n2 = bv.n[s2];
    const int r0 = ((lb * CL) + rank) * 8;
    const int rb = min(8, n2 - r0);
    if (rb <= 0) return false;
    b0 = reinterpret_cast<uintptr_t>(bv.A + bv.offA[s2] + int64_t(r0) * n2);
    b1 = b0 + uintptr_t(rb) * uintptr_t(n2) * 8u;
    return true;
  };
  auto stage_issue = [&](int it) {   // the pivot warp, all lanes
    const int s2 = bv.list[it];
    unsigned bytes = 0;
    uintptr_t i0 = 0, b0, b1;
    if (lane < LP / 8 && block_span(s2, lane, b0, b1)) {
      i0 = (b0 + 15) & ~uintptr_t(15);
      const uintptr_t i1 = b1 & ~uintptr_t(15);
      if (i1 > i0) bytes = unsigned(i1 - i0);
    }
    unsigned tot = bytes;
#pragma unroll
    for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0) mbar_expect_tx(bar, tot);
    __syncwarp();
    if (bytes) {
      const int shift = int((b0 >> 3) & 1);
      bulk_g2s(stage + lane * S::SLOT + 2 * shift, reinterpret_cast<const void*>(i0), bytes, bar);
    }
  };
  // the ends of each block that the aligned copy leaves out, by plain loads
  auto stage_ends = [&](int s2) {    // the pivot warp
    uintptr_t b0, b1;
    if (lane < LP / 8 && block_span(s2, lane, b0, b1)) {
      const int shift = int((b0 >> 3) & 1);
      double* slot = stage + lane * S::SLOT + shift;
      const double* g = reinterpret_cast<const double*>(b0);
      const int64_t ne = int64_t((b1 - b0) >> 3);
      if (shift) slot[0] = g[0];                                   // head: b0 not 16-byte aligned
      if ((b1 & 15) && (ne > 1 || !shift)) slot[ne - 1] = g[ne - 1];   // tail: b1 not 16-byte aligned
    }
  };
  if (!tile) {
    if (lane == 0) {
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncwarp();
  }
  __syncthreads();
  if (!tile && cid < cnt) stage_issue(cid);
  unsigned sphase = 0;

  int parity = 0;   // the certificate flags alternate buffers: a peer is at most one item ahead
  for (int item = cid; item < cnt; item += ncl, parity ^= 1) {
    const int s = bv.list[item];
    const int n = bv.n[s];

    // ---- this matrix's rows from the staging slots into registers (identity
    // padding), and the certificate's partial sums
    const bool stalled = !mbar_wait(bar, sphase, kStageWaitPolls);
    sphase ^= 1;
    if (!tile && !stalled) stage_ends(s);
    __syncthreads();
    double* red = sm;   // [CT][LP] partial off-diagonal sums, over the panel buffers
    double* dg = sm + S::off_dg;
    bool zok = !stalled;
    if (tile) {
      int shift[TR];
#pragma unroll
      for (int i = 0; i < TR; ++i) {
        uintptr_t b0, b1;
        const int lb = (tr + RT * i) >> 3;
        shift[i] = block_span(s, lb, b0, b1) ? int((b0 >> 3) & 1) : 0;
      }
#pragma unroll
      for (int i = 0; i < TR; ++i) {
        const int r = grow(i);
        const double* slot = stage + ((tr + RT * i) >> 3) * S::SLOT + shift[i] + ((tr + RT * i) & 7) * n;
        double part = 0.0;
#pragma unroll
        for (int j = 0; j < TC; ++j) {
          const int c = tc + CT * j;
          const double a = (r < n && c < n) ? slot[c] : ((r == c) ? 1.0 : 0.0);
          W[i][j] = a;
          if (c == r) {
            dg[tr + RT * i] = a;
          } else {
            zok &= (a <= 0.0);    // false for NaN
            part += fabs(a);
          }
        }
        red[tc * LP + tr + RT * i] = part;
      }
    }
    __syncthreads();
    bool rok = true;
    for (int lr = tid; lr < LP; lr += S::NTH) {
      double off = 0.0;
      for (int t = 0; t < CT; ++t) off += red[t * LP + lr];
      const double d = dg[lr];
      rok &= (d > 0.0) && (d < INFINITY) && (off * (1.0 + 0x1p-40) <= (1.0 - kCertMargin) * d);
    }
    const int cert_cta = __syncthreads_and(int(zok && rok));
    const int stall_cta = __syncthreads_or(int(stalled));
    int cert = cert_cta, stall = stall_cta;
    if (CL > 1) {
      cg::cluster_group cl = cg::this_cluster();
      double* okf = sm + S::off_ok + 8 * parity;
      if (tid == 0) {
        for (int pr = 0; pr < CL; ++pr)
          cl.map_shared_rank(okf, pr)[rank] = double(cert_cta) + 2.0 * double(stall_cta);
      }
      cluster_barrier<CL>();
      for (int pr = 0; pr < CL; ++pr) {
        const int f = int(okf[pr]);
        cert &= f & 1;
        stall |= f >> 1;
      }
    }
    if (stall) {
      // a staging copy never completed: report it, give the copy a second
      // bounded wait, and leave (no CTA of the cluster issues more copies)
      if (rank == 0 && tid == 0) bv.status[s] = kStageTimeout;
      if (stalled) mbar_wait(bar, sphase ^ 1, kStageWaitPolls);
      cluster_barrier<CL>();
      return;
    }
    // the staging slots are free again: fetch the next matrix during this one
    if (!tile && item + ncl < cnt) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      stage_issue(item + ncl);
    }
    if (!cert) {
      if (rank == 0 && tid == 0) {
        const int cls = ca.xcls[s];
        const int slot = atomicAdd(ca.fb_count + cls, 1);
        ca.fb_list[ca.fb_off[cls] + slot] = s;
      }
      __syncthreads();
      continue;
    }

    // ---- prologue: the first pivot block and its inverse
    if (tile) {
      publish(0);
      share_row_panel(0);
    }
    cluster_barrier<CL>();
    if (!tile && rank == 0) {
      const double* RowPT = bufp(0) + S::off_RowPT;
      const int q = lane >> 2, h = lane & 3;
      pivot_inverse(0, RowPT[(2 * h) * SP + q], RowPT[(2 * h + 1) * SP + q]);
    }
    cluster_barrier<CL>();

    // ---- blocked Gauss-Jordan, one 8 x 8 pivot block per step
    for (int kblk = 0; kblk < NBLK; ++kblk) {
      double* B = bufp(kblk);
      const double* RowPT = B + S::off_RowPT;
      double* RowNT = B + S::off_RowNT;
      const double* ColP = B + S::off_ColP;
      const double* Dinv = B + S::off_Dinv;
      const int kb = 8 * kblk;

      if (kblk > 0) {
        if (tile) {
          publish(kblk);
          share_row_panel(kblk);
        }
        cluster_barrier<CL>();   // also orders the pivot warp's D^-1 of this block
      }

      // S3: R' = D^-1 R outside K, I + D^-1 on K's columns; a thread always
      // forms entries of the same panel row q, so it reads row q of D^-1 once
      if (tile) {
        const int q = tid & 7;
        double dv[8];
#pragma unroll
        for (int p = 0; p < 8; ++p) dv[p] = Dinv[q * SP + p];
#pragma unroll
        for (int e0 = 0; e0 < 8 * P; e0 += NT) {
          const int e = e0 + tid;
          if (8 * P % NT != 0 && e >= 8 * P) break;
          const int c = e >> 3;
          double val = 0.0;
#pragma unroll
          for (int p = 0; p < 8; ++p) val = fma(dv[p], RowPT[c * SP + p], val);
          const int ck = c - kb;
          const bool inK = unsigned(ck) < 8u;
          const double kv = Dinv[q * SP + (inK ? ck : 0)] + ((q == ck) ? 1.0 : 0.0);
          RowNT[c * SP + q] = inK ? kv : val;
        }
      }
      __syncthreads();

      if (tile) {
        // S4: W -= C' R'
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          double cp[TR], rn[TC];
#pragma unroll
          for (int i = 0; i < TR; ++i) cp[i] = ColP[(tr + RT * i) * SP + q];
#pragma unroll
          for (int j = 0; j < TC; ++j) rn[j] = RowNT[(tc + CT * j) * SP + q];
#pragma unroll
          for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) W[i][j] = fma(-cp[i], rn[j], W[i][j]);
        }
      } else if (kblk + 1 < NBLK && rank == (kblk + 1) % CL) {
        // the next pivot block, updated exactly as its holders update it, then inverted
        const int q = lane >> 2, h = lane & 3;
        const int lr = ((kblk + 1) / CL) * 8 + q;     // local row of the next block's row q
        const double* Dn = B + S::off_Dnext;
        double d0 = Dn[q * SP + 2 * h], d1 = Dn[q * SP + 2 * h + 1];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const double cpk = ColP[lr * SP + k];
          d0 = fma(-cpk, RowNT[(kb + 8 + 2 * h) * SP + k], d0);
          d1 = fma(-cpk, RowNT[(kb + 9 + 2 * h) * SP + k], d1);
        }
        pivot_inverse(kblk + 1, d0, d1);
      }
    }

    // ---- store N^-1
    if (tile) {
      double* __restrict__ Og = bv.out + bv.offA[s];
#pragma unroll
      for (int i = 0; i < TR; ++i) {
        const int r = grow(i);
        if (r < n) {
#pragma unroll
          for (int j = 0; j < TC; ++j) {
            const int c = tc + CT * j;
            if (c < n) Og[int64_t(r) * n + c] = W[i][j];
          }
        }
      }
    }
    if (rank == 0 && tid == 0) {
      bv.status[s] = kOk;
      if (bv.diag) bv.diag[s] = 0;
    }
    // the next item reuses the panel buffers: every CTA of the cluster is done
    // with this one (including remote writes of its last pivot inverse)
    cluster_barrier<CL>();
  }
}

}  // namespace ss
