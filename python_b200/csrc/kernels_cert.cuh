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
//     1/4 <= a_rr <= 4,  a_rc <= 0 (c != r),  sum_{c != r} |a_rc| * (1 + 2^-40) <= (1 - tau) a_rr
// for every row r, tau = kCertMargin, with every entry finite.  The bound on
// the diagonal is the fused update's (below): it adds I to D^-1 and takes it
// from the column panel, which is accurate relative to unit scale only; a row
// scaled by 2^e loses about e bits (rows at 2^+-20: 2.7e-10 from the true
// inverse), so matrices of other scales take the exact path.  Measured against
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
// factorisation, spread over the tile warps of one CTA or of a cluster of CL
// CTAs (one SM each).  Rows go to the cluster's CTAs in blocks of 8 (block b to
// CTA b % CL).  A CTA's rows and all columns form 8 x 8 sub-blocks; tile warp
// (wr, wc) of a WGR x WGC warp grid owns local row blocks wr + WGR i and column
// blocks wc + WGC j, each sub-block held as the accumulator fragment of the
// FP64 tensor-core MMA (mma.sync m8n8k4 f64: lane l holds row l/4, columns
// 2(l%4) and 2(l%4)+1).  Each CTA also runs one pivot warp that holds no tile.
// Every block step moves only the two panels through shared memory:
//   S1  the warps holding K's rows write R (transposed, RowPT[c][q]) into
//       the shared memory of every CTA of the cluster (remote stores into
//       distributed shared memory, so that S3 reads are local); the warps
//       holding K's columns write
//       -C' (ColPN[r][q] = I - C on D's diagonal, -C elsewhere) locally; the
//       holder of the next pivot block writes its current values (Dnext);
//       then a cluster barrier;
//   S3  R' = D^-1 R, two MMAs per 8-column block: with a single row of tile
//       warps (WGR = 1) each warp forms R' for its own columns in registers
//       (computed transposed, so that the accumulator is already the update's
//       B operand); otherwise the tile warps share the columns and write R'
//       to shared memory (RowNT[c][q]), followed by a barrier;
//   S4  every tile warp adds (-C') R' into each of its sub-blocks, two MMAs per
//       sub-block from one operand load per row and per column block, while
//       the pivot warp of the CTA that owns the next block brings Dnext up to
//       date with the same MMAs in the same order and inverts it (8 x 8, the
//       accumulator fragment's two entries per lane, shuffles; on one-CTA
//       classes an FP32 elimination refined by FP64 Newton steps), writing
//       D^-1 of the next step into every CTA of the cluster.
// So the serial 8 x 8 inverse overlaps the bulk update, and a step costs one
// cluster barrier (plus one CTA barrier when R' goes through shared memory).
// A matrix of order n takes ceil(n / 8) steps: the blocks beyond it hold only
// the identity padding, which no step would change.  Panel rows hold 8 values
// at a stride of SP = 12 doubles: the operand fragments (8 panel rows x 4
// values per load) then fall on distinct banks.  The row panel, -C', D^-1 and
// Dnext are double-buffered by step parity.  B200's FP64 tensor-core MMA runs
// at the FP64 FMA rate (both ~37 TF/s here); it is used for its eight-fold
// fewer issued instructions and its operand reuse across a warp, and it keeps
// the FMA pipe free for the pivot warp's chain.
// Staging: the rows a CTA holds arrive in shared memory by 1-D TMA bulk copies
// (cp.async.bulk, one per 8-row block, completing on an mbarrier), issued for
// the NEXT matrix as soon as the current one has moved into registers, so the
// HBM latency of a matrix overlaps the factorisation of the one before.  A bulk
// copy needs 16-byte aligned ends: the aligned interior of each block is
// copied, and the at most two 8-byte ends are read by plain loads, so nothing
// outside the caller's matrix is touched.
#pragma once
#include <cooperative_groups.h>

#include "ss_common.cuh"

namespace ss {

constexpr double kCertMargin = 1.0e-5;   // relative row-dominance margin of the certificate
constexpr double kCertDiagLo = 0.25, kCertDiagHi = 4.0;   // the certificate's range of a_rr

// Fallback lists of the certified launches: systems that fail the certificate
// are appended, per exact-path size class, for the GSL-exact kernels.
struct CertArgs {
  const int* xcls;     // [nsys] exact-path class list of each system
  const int* fb_off;   // [classes] start of each class's list in fb_list
  int* fb_list;        // the lists
  int* fb_count;       // [classes] entries appended (zeroed before the launch)
};

// The macro-atom epilogue fused into the certified kernel (calc_matom_matrix,
// source/macro_accelerate.c:325-334, and the running total of
// matom_deactivation_from_matrix, :995-1008): with R set, the kernel writes
// B = N^-1 diag(R) (one rounding per product, a_inverse * R as the reference
// forms it) instead of N^-1, and with C set also the row running totals
// C[r][c] = B[r][0] + ... + B[r][c], added left to right, one rounding per
// addition.  R of system s starts at offv[s].
struct CertEpi {
  const int64_t* offv = nullptr;
  const double* R = nullptr;
  double* C = nullptr;
};

// P: padded order; WGR x WGC: tile-warp grid of one CTA; CL: CTAs per matrix (a
// cluster); MINB: CTAs per SM asked of the register allocator; STAGE: rows
// arrive through the TMA staging slots (else straight from global memory into
// registers, which leaves shared memory for more CTAs per SM).
template <int P_, int WGR_, int WGC_, int CL_, int MINB_, bool STAGE_ = true>
struct CgjShape {
  static constexpr bool STAGE = STAGE_;
  static constexpr int P = P_, WGR = WGR_, WGC = WGC_, CL = CL_;
  static constexpr int NW = WGR * WGC;     // tile warps
  static constexpr int NT = 32 * NW;       // tile threads
  static constexpr int NTH = NT + 32;      // with the pivot warp
  static constexpr int LP = P / CL;        // rows held by one CTA
  static constexpr int LB = LP / 8;        // local 8-row blocks
  static constexpr int CBK = P / 8;        // 8-column blocks
  static constexpr int WR = LB / WGR;      // row blocks per tile warp
  static constexpr int WC = CBK / WGC;     // column blocks per tile warp
  static constexpr int MINB = MINB_;
  static constexpr int SP = 12;            // stride of a panel row (8 values)
  // shared memory, in doubles, per panel buffer (two buffers, by step parity)
  static constexpr int off_RowPT = 0;                   // [P][SP]
  static constexpr int off_ColP = SP * P;               // [LP][SP]  -C'
  static constexpr int off_Dinv = SP * P + SP * LP;     // [8][SP]
  static constexpr int off_Dnext = off_Dinv + 8 * SP;   // [8][SP]
  static constexpr int buf = off_Dnext + 8 * SP;
  // R' has one buffer: S3 writes it after a step's first barrier and the last
  // reader (S4 and the pivot warp) is done before the next step's first barrier.
  // A single row of tile warps (WGR = 1) keeps R' in registers instead.
  static constexpr bool REGR = (WGR_ == 1);
  static constexpr int off_RowNT = 2 * buf;             // [P][SP]
  static constexpr int off_dg = off_RowNT + (REGR ? 0 : SP * P);   // [LP] diagonal of each local row
  static constexpr int off_ok = off_dg + LP;            // [2][8] certificate of each CTA, by item parity
  static constexpr int off_bar = off_ok + 16;           // the staging mbarrier (8 bytes)
  static constexpr int SLOT = 8 * P + 2;                // doubles per staged 8-row block (+ alignment shift)
  static constexpr int off_stage = off_bar + 2;         // [LB][SLOT], 16-byte aligned
  static constexpr int n_dbl = off_stage + (STAGE ? LB * SLOT : 0);
  static constexpr size_t dyn_smem = size_t(n_dbl) * 8;
  static_assert(P % (8 * CL) == 0 && LB % WGR == 0 && CBK % WGC == 0, "whole sub-block tiles");
  static_assert(NTH <= 1024, "one CTA");
  static_assert(WGC * LP <= off_Dinv, "certificate partials leave D^-1 and Dnext free (pivot scratch)");
  static_assert(CL >= 1 && CL <= 8, "portable cluster sizes");
  static_assert(off_stage % 2 == 0 && SLOT % 2 == 0, "16-byte aligned staging slots");
  static_assert(buf % 2 == 0 && off_dg % 2 == 0, "16-byte aligned buffers");
  static_assert(!STAGE || LB <= 32, "one lane of the pivot warp issues each block's copy");
  static_assert(dyn_smem <= 232448, "one CTA's shared memory");
  static_assert(((LP + 31) / 32) * 32 * 33 <= off_dg && (LP + 31) / 32 <= NW,
                "the running-total tiles fit the panel buffers, one tile warp per 32 rows");
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

// d[0..1] += A (8 x 4, lane l: row l/4, column l%4) * B (4 x 8, lane l: row
// l%4, column l/4), FP64 on the tensor cores; d is the accumulator fragment
// (lane l: row l/4, columns 2(l%4) and 2(l%4)+1).
__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// In-place Gauss-Jordan inverse of the 8 x 8 pivot block by one warp, without
// pivoting.  Lane l holds D[l/4][2(l%4)] in d0 and D[l/4][2(l%4)+1] in d1 (the
// accumulator fragment's layout).  (Measured alone on an SM: ~910 cycles per
// call; a variant taking two pivots at a time through 2 x 2 determinants
// needed more shuffles and took ~1250.)
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

// The same elimination in FP32, with the hardware's approximate reciprocal:
// a starting point for warp_inv8_refined, on the FP32 pipe.
__device__ __forceinline__ void warp_inv8_f32(float& d0, float& d1, int lane) {
  const int q = lane >> 2, h = lane & 3;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int kh = k >> 1;
    const float colv = (k & 1) ? d1 : d0;
    const float dkk = __shfl_sync(0xffffffffu, colv, 4 * k + kh);
    const float f = __shfl_sync(0xffffffffu, colv, 4 * q + kh);
    const float rk0 = __shfl_sync(0xffffffffu, d0, 4 * k + h);
    const float rk1 = __shfl_sync(0xffffffffu, d1, 4 * k + h);
    float piv;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(piv) : "f"(dkk));
    const float nk0 = (2 * h == k) ? piv : rk0 * piv;
    const float nk1 = (2 * h + 1 == k) ? piv : rk1 * piv;
    if (q == k) {
      d0 = nk0;
      d1 = nk1;
    } else {
      d0 = fmaf(-f, nk0, (2 * h == k) ? 0.0f : d0);
      d1 = fmaf(-f, nk1, (2 * h + 1 == k) ? 0.0f : d1);
    }
  }
}

// |x| as the ordered high word of a double (sign cleared; NaN and Inf above
// every finite value), for warp-wide maxima on the integer pipe
__device__ __forceinline__ unsigned abs_hi(double x) {
  return unsigned(__double2hiint(x)) & 0x7fffffffu;
}
__device__ __forceinline__ double neg_bits(double x) {   // -x by its sign bit
  return __longlong_as_double(__double_as_longlong(x) ^ (1ll << 63));
}

// The 8 x 8 inverse of warp_inv8 with little FP64 work on its serial path: the
// FP32 elimination above gives X, then Newton steps X <- X + X (I - D X) in
// FP64 on the tensor cores (two MMAs for the residual, two for the update)
// until the residual's largest entry is below 2^-27, after which the last
// update leaves X at FP64 rounding.  A block whose first residual is 1/4 or
// more (a badly conditioned or badly scaled D, an FP32 overflow, NaN) or that
// has not converged after four steps is inverted by warp_inv8 instead.  Where
// the pivot warp's chain is a step's critical path while the tile warps keep
// the FP64 pipe busy, this moves all but ~12 of its ~64 FP64 instructions to
// the FP32 pipe.  scrD and scrX are two free 8 x SP panels of
// shared memory (row-major, stride SP) for the operand transposes.
template <int SP>
__device__ __forceinline__ void warp_inv8_refined(double& d0, double& d1, int lane, double* scrD,
                                                  double* scrX) {
  const int g = lane >> 2, t = lane & 3;
  constexpr unsigned kHiQuarter = 1021u << 20;    // |e| >= 2^-2
  constexpr unsigned kHiConverged = 996u << 20;   // |e| <  2^-27
  float f0 = __double2float_rn(d0), f1 = __double2float_rn(d1);
  warp_inv8_f32(f0, f1, lane);
  double x0 = double(f0), x1 = double(f1);
  __syncwarp();   // earlier reads of the scratch panels by this warp
  scrD[g * SP + 2 * t] = neg_bits(d0);
  scrD[g * SP + 2 * t + 1] = neg_bits(d1);
  __syncwarp();
  const double na0 = scrD[g * SP + t], na1 = scrD[g * SP + 4 + t];   // -D, A operand
  bool ok = false;
#pragma unroll 1
  for (int it = 0; it < 4; ++it) {
    scrX[g * SP + 2 * t] = x0;
    scrX[g * SP + 2 * t + 1] = x1;
    __syncwarp();
    const double xb0 = scrX[t * SP + g], xb1 = scrX[(4 + t) * SP + g];   // X, B operand
    const double xa0 = scrX[g * SP + t], xa1 = scrX[g * SP + 4 + t];     // X, A operand
    __syncwarp();
    double e[2] = {(g == 2 * t) ? 1.0 : 0.0, (g == 2 * t + 1) ? 1.0 : 0.0};
    dmma_884(e, na0, xb0);
    dmma_884(e, na1, xb1);
    const unsigned em = __reduce_max_sync(0xffffffffu, max(abs_hi(e[0]), abs_hi(e[1])));
    if (em >= kHiQuarter) break;
    scrX[g * SP + 2 * t] = e[0];
    scrX[g * SP + 2 * t + 1] = e[1];
    __syncwarp();
    const double eb0 = scrX[t * SP + g], eb1 = scrX[(4 + t) * SP + g];   // E, B operand
    __syncwarp();
    double xn[2] = {x0, x1};
    dmma_884(xn, xa0, eb0);
    dmma_884(xn, xa1, eb1);
    x0 = xn[0];
    x1 = xn[1];
    if (em < kHiConverged) {
      ok = true;
      break;
    }
  }
  if (ok) {
    d0 = x0;
    d1 = x1;
  } else {
    warp_inv8(d0, d1, lane);
  }
}

template <int P, int WGR, int WGC, int CL, int MINB, bool STAGE = true>
__global__ void __launch_bounds__(32 * WGR * WGC + 32, MINB)
cgj_inverse_kernel(BatchView bv, CertArgs ca, CertEpi ep) {
  using S = CgjShape<P, WGR, WGC, CL, MINB, STAGE>;
  constexpr int NW = S::NW, WR = S::WR, WC = S::WC, LP = S::LP, LB = S::LB, CBK = S::CBK;
  constexpr int SP = S::SP, NBLK = P / 8;
  extern __shared__ __align__(16) double sm[];
  namespace cg = cooperative_groups;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;      // fragment row, column pair
  const bool tile = warp < NW;                // the last warp is the pivot warp
  const int wr = warp / WGC, wc = warp % WGC;  // meaningful for tile warps
  const int rank = (CL > 1) ? int(cluster_rank()) : 0;
  const int cid = blockIdx.x / CL, ncl = gridDim.x / CL;
  const int cnt = batch_count(bv);

  // local row (in this CTA) and global row of this lane's row in sub-block row i,
  // global column of its column e in sub-block column j
  auto lrow = [&](int i) -> int { return (wr + WGR * i) * 8 + g; };
  auto grow = [&](int i) -> int { return ((wr + WGR * i) * CL + rank) * 8 + g; };
  auto gcol = [&](int j, int e) -> int { return (wc + WGC * j) * 8 + 2 * t + e; };
  auto bufp = [&](int kblk) -> double* { return sm + (kblk & 1) * S::buf; };
  double W[WR][WC][2];
  // block steps of the current matrix: those whose pivot block holds no row
  // of it would only carry the identity padding along, so they are skipped
  int nbe = NBLK;

  // S1 of block kblk: the old row panel, -C' and the next pivot block's values
  // REGR classes on a cluster push each row panel ahead (during the update of
  // the step before), so publish then leaves it out
  constexpr bool kEarlyRows = S::REGR && (CL > 1);
  auto publish = [&](int kblk) {
    double* B = bufp(kblk);
    double* RowPT = B + S::off_RowPT;
    double* ColP = B + S::off_ColP;
    const int kb = 8 * kblk;
    const int lbK = kblk / CL;
    if (!(kEarlyRows && kblk > 0) && rank == kblk % CL && wr == lbK % WGR) {
      const int iK = lbK / WGR;
#pragma unroll
      for (int j = 0; j < WC; ++j) {
        double v0 = W[0][j][0], v1 = W[0][j][1];
#pragma unroll
        for (int i = 1; i < WR; ++i)
          if (i == iK) {
            v0 = W[i][j][0];
            v1 = W[i][j][1];
          }
        RowPT[gcol(j, 0) * SP + g] = v0;
        RowPT[gcol(j, 1) * SP + g] = v1;
        if (CL > 1) {
          // the row panel also goes straight into the other CTAs' shared memory,
          // so that every CTA reads its S3 operands locally
#pragma unroll
          for (int pr = 0; pr < CL; ++pr) {
            if (pr == rank) continue;
            double* rp = cg::this_cluster().map_shared_rank(RowPT, pr);
            rp[gcol(j, 0) * SP + g] = v0;
            rp[gcol(j, 1) * SP + g] = v1;
          }
        }
      }
    }
    if (wc == kblk % WGC) {
      const int jK = kblk / WGC;
#pragma unroll
      for (int i = 0; i < WR; ++i) {
        double v0 = W[i][0][0], v1 = W[i][0][1];
#pragma unroll
        for (int j = 1; j < WC; ++j)
          if (j == jK) {
            v0 = W[i][j][0];
            v1 = W[i][j][1];
          }
        const int r = grow(i);
        // with R' in registers the columns are stored in slice order (column
        // 2t + e at 4e + t, see S3)
        const int p0 = S::REGR ? t : 2 * t, p1 = S::REGR ? 4 + t : 2 * t + 1;
        ColP[lrow(i) * SP + p0] = ((r == kb + 2 * t) ? 1.0 : 0.0) - v0;
        ColP[lrow(i) * SP + p1] = ((r == kb + 2 * t + 1) ? 1.0 : 0.0) - v1;
      }
    }
    if (kblk + 1 < nbe) {
      const int k1 = kblk + 1, lbK1 = k1 / CL;
      if (rank == k1 % CL && wr == lbK1 % WGR && wc == k1 % WGC) {
        const int i1 = lbK1 / WGR, j1 = k1 / WGC;
        double v0 = W[0][0][0], v1 = W[0][0][1];
#pragma unroll
        for (int i = 0; i < WR; ++i)
#pragma unroll
          for (int j = 0; j < WC; ++j)
            if (i == i1 && j == j1) {
              v0 = W[i][j][0];
              v1 = W[i][j][1];
            }
        B[S::off_Dnext + g * SP + 2 * t] = v0;
        B[S::off_Dnext + g * SP + 2 * t + 1] = v1;
      }
    }
  };

  // the pivot warp: D^-1 of block kblk from the 8 x 8 values d0, d1
  // (accumulator layout), written into every CTA's buffer of that block
  auto pivot_inverse = [&](int kblk, double d0, double d1) {
    // One CTA per matrix: the FP32 start and FP64 Newton steps (orders 57-64
    // +15 %, 121-128 +5 %); on a cluster the FP64 elimination, which measured
    // 0-5 % faster there.  Scratch: this block's D^-1 panel (written last) and
    // the other buffer's Dnext panel (read by this warp already; rewritten two
    // steps later)
    if constexpr (CL == 1)
      warp_inv8_refined<SP>(d0, d1, lane, bufp(kblk + 1) + S::off_Dnext, bufp(kblk) + S::off_Dinv);
    else
      warp_inv8(d0, d1, lane);
    double* Dinv = bufp(kblk) + S::off_Dinv;
    Dinv[g * SP + 2 * t] = d0;
    Dinv[g * SP + 2 * t + 1] = d1;
    if (CL > 1) {
      cg::cluster_group cl = cg::this_cluster();
#pragma unroll
      for (int pr = 0; pr < CL; ++pr) {
        if (pr == rank) continue;
        double* rp = cl.map_shared_rank(Dinv, pr);
        rp[g * SP + 2 * t] = d0;
        rp[g * SP + 2 * t + 1] = d1;
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
  // the ends of each block that the aligned copy leaves out: read with plain
  // loads when the copy is issued, kept in the issuing lane's registers, and
  // written into the slot once the copy has landed
  double head_v = 0.0, tail_v = 0.0;
  auto stage_issue = [&](int it) {   // the pivot warp, all lanes
    const int s2 = bv.list[it];
    unsigned bytes = 0;
    uintptr_t i0 = 0, b0 = 0, b1 = 0;
    if (lane < LB && block_span(s2, lane, b0, b1)) {
      i0 = (b0 + 15) & ~uintptr_t(15);
      const uintptr_t i1 = b1 & ~uintptr_t(15);
      if (i1 > i0) bytes = unsigned(i1 - i0);
      const double* gp = reinterpret_cast<const double*>(b0);
      const int64_t ne = int64_t((b1 - b0) >> 3);
      head_v = gp[0];
      tail_v = gp[ne - 1];
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
  auto stage_ends = [&](int s2) {    // the pivot warp
    uintptr_t b0, b1;
    if (lane < LB && block_span(s2, lane, b0, b1)) {
      const int shift = int((b0 >> 3) & 1);
      double* slot = stage + lane * S::SLOT + shift;
      const int64_t ne = int64_t((b1 - b0) >> 3);
      if (shift) slot[0] = head_v;                                     // head: b0 not 16-byte aligned
      if ((b1 & 15) && (ne > 1 || !shift)) slot[ne - 1] = tail_v;       // tail: b1 not 16-byte aligned
    }
  };
  if (STAGE && !tile) {
    if (lane == 0) {
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncwarp();
  }
  __syncthreads();
  if (STAGE && !tile && cid < cnt) stage_issue(cid);
  unsigned sphase = 0;

  int parity = 0;   // the certificate flags alternate buffers: a peer is at most one item ahead
  for (int item = cid; item < cnt; item += ncl, parity ^= 1) {
    const int s = bv.list[item];
    const int n = bv.n[s];
    nbe = (n + 7) / 8;

    // ---- this matrix's rows from the staging slots into registers (identity
    // padding), and the certificate's partial sums
    bool stalled = false;
    if (STAGE) {
      stalled = !mbar_wait(bar, sphase, kStageWaitPolls);
      sphase ^= 1;
      if (!tile && !stalled) stage_ends(s);
    }
    __syncthreads();
    // the pivot warp of the CTA holding block 0 inverts D(0) straight from the
    // staging slots while the tile warps check the certificate (wasted, and
    // harmless, if the matrix fails it)
    if (!tile && rank == 0 && !stalled) {
      double d[2];
      if (STAGE) {
        uintptr_t b0, b1;
        const int shift = block_span(s, 0, b0, b1) ? int((b0 >> 3) & 1) : 0;
        const double* slot = stage + shift + g * n;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = 2 * t + e;
          d[e] = (g < n && c < n) ? slot[c] : ((g == c) ? 1.0 : 0.0);
        }
      } else {
        const double* Ag = bv.A + bv.offA[s];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = 2 * t + e;
          d[e] = (g < n && c < n) ? __ldg(Ag + int64_t(g) * n + c) : ((g == c) ? 1.0 : 0.0);
        }
      }
      pivot_inverse(0, d[0], d[1]);
    }
    double* red = sm;   // [WGC][LP] partial off-diagonal sums, over the panel buffers
    double* dg = sm + S::off_dg;
    bool zok = !stalled;
    if (tile && !STAGE) {
      // every load issued unconditionally (padding entries read A[0][0]), so
      // all of a lane's loads are in flight at once
      const double* __restrict__ Ag = bv.A + bv.offA[s];
#pragma unroll
      for (int i = 0; i < WR; ++i) {
        const int r = grow(i);
#pragma unroll
        for (int j = 0; j < WC; ++j)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int c = gcol(j, e);
            W[i][j][e] = __ldg(Ag + ((r < n && c < n) ? int64_t(r) * n + c : 0));
          }
      }
    }
    if (tile) {
#pragma unroll
      for (int i = 0; i < WR; ++i) {
        uintptr_t b0, b1;
        const int lb = wr + WGR * i;
        const int shift = (STAGE && block_span(s, lb, b0, b1)) ? int((b0 >> 3) & 1) : 0;
        const double* slot = stage + lb * S::SLOT + shift + g * n;
        const int r = grow(i);
        double part = 0.0;
#pragma unroll
        for (int j = 0; j < WC; ++j)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int c = gcol(j, e);
            const double a = (r < n && c < n) ? (STAGE ? slot[c] : W[i][j][e]) : ((r == c) ? 1.0 : 0.0);
            W[i][j][e] = a;
            if (c == r) {
              dg[lrow(i)] = a;
            } else {
              zok &= (a <= 0.0);    // false for NaN
              part += fabs(a);
            }
          }
        part += __shfl_xor_sync(0xffffffffu, part, 1);
        part += __shfl_xor_sync(0xffffffffu, part, 2);
        if (t == 0) red[wc * LP + lrow(i)] = part;
      }
    }
    __syncthreads();
    bool rok = true;
    for (int lr = tid; lr < LP; lr += S::NTH) {
      double off = 0.0;
      for (int q = 0; q < WGC; ++q) off += red[q * LP + lr];
      const double d = dg[lr];
      rok &= (d >= kCertDiagLo) && (d <= kCertDiagHi) && (off * (1.0 + 0x1p-40) <= (1.0 - kCertMargin) * d);
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
      if (STAGE && stalled) mbar_wait(bar, sphase ^ 1, kStageWaitPolls);
      cluster_barrier<CL>();
      return;
    }
    // the staging slots are free again: fetch the next matrix during this one
    if (STAGE && !tile && item + ncl < cnt) {
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

    // ---- prologue: the first panels (D(0)^-1 is already in place)
    if (tile) publish(0);
    cluster_barrier<CL>();

    // ---- blocked Gauss-Jordan, one 8 x 8 pivot block per step
    for (int kblk = 0; kblk < nbe; ++kblk) {
      double* B = bufp(kblk);
      const double* RowPT = B + S::off_RowPT;   // written into every CTA by the owner
      double* RowNT = sm + S::off_RowNT;
      const double* ColP = B + S::off_ColP;
      const double* Dinv = B + S::off_Dinv;
      const int kb = 8 * kblk;

      if (kblk > 0) {
        if (tile) publish(kblk);
        cluster_barrier<CL>();   // also orders the pivot warp's D^-1 of this block
      }

      if constexpr (S::REGR) {
        // S3 in registers: each tile warp forms R' (D^-1 R outside K, I + D^-1
        // on K's columns) for its own columns, transposed (R'^T = R^T D^-T):
        // the accumulator gives each lane R'[2t][c] and R'[2t + 1][c] of column
        // c = 8 cb + g, the B operand of the update for the k-slices {2t} and
        // {2t + 1}; the column panel is stored in that slice order.  No R'
        // buffer, so no barrier between S3 and S4.
        const double d0 = Dinv[g * SP + t], d1 = Dinv[g * SP + 4 + t];   // D^-T, B operand
        if (tile) {
          double bf[WC][2];
#pragma unroll
          for (int j = 0; j < WC; ++j) {
            const int cb = wc + WGC * j;
            if (cb == kblk) {
              bf[j][0] = Dinv[(2 * t) * SP + g] + ((g == 2 * t) ? 1.0 : 0.0);
              bf[j][1] = Dinv[(2 * t + 1) * SP + g] + ((g == 2 * t + 1) ? 1.0 : 0.0);
            } else {
              bf[j][0] = 0.0;
              bf[j][1] = 0.0;
              dmma_884(bf[j], RowPT[(cb * 8 + g) * SP + t], d0);
              dmma_884(bf[j], RowPT[(cb * 8 + g) * SP + 4 + t], d1);
            }
          }
          // S4: W += (-C') R', two MMAs per sub-block.  On a cluster, the CTA
          // holding the next row block updates that block first and pushes it
          // as the next row panel into every CTA, so that the remote stores
          // complete during the rest of the update rather than at the barrier
          const bool early = kEarlyRows && kblk + 1 < nbe && rank == (kblk + 1) % CL;
          const int iK1 = (kblk + 1) / CL;   // its local block (one row of tile warps)
          if (early) {
            double* RowN = bufp(kblk + 1) + S::off_RowPT;
#pragma unroll
            for (int i = 0; i < WR; ++i)
              if (i == iK1) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                  const double a = ColP[lrow(i) * SP + 4 * h + t];
#pragma unroll
                  for (int j = 0; j < WC; ++j) dmma_884(W[i][j], a, bf[j][h]);
                }
#pragma unroll
                for (int j = 0; j < WC; ++j) {
#pragma unroll
                  for (int pr = 0; pr < CL; ++pr) {
                    double* rp = (pr == rank) ? RowN : cg::this_cluster().map_shared_rank(RowN, pr);
                    rp[gcol(j, 0) * SP + g] = W[i][j][0];
                    rp[gcol(j, 1) * SP + g] = W[i][j][1];
                  }
                }
              }
          }
#pragma unroll
          for (int i = 0; i < WR; ++i)
            if (!(early && i == iK1)) {
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const double a = ColP[lrow(i) * SP + 4 * h + t];
#pragma unroll
                for (int j = 0; j < WC; ++j) dmma_884(W[i][j], a, bf[j][h]);
              }
            }
        } else if (kblk + 1 < nbe && rank == (kblk + 1) % CL) {
          // the next pivot block, updated exactly as its holder updates it
          // (R' of its columns formed here), then inverted
          const int lr0 = ((kblk + 1) / CL) * 8;
          const double* Dn = B + S::off_Dnext;
          double r1[2] = {0.0, 0.0};
          dmma_884(r1, RowPT[((kblk + 1) * 8 + g) * SP + t], d0);
          dmma_884(r1, RowPT[((kblk + 1) * 8 + g) * SP + 4 + t], d1);
          double d[2] = {Dn[g * SP + 2 * t], Dn[g * SP + 2 * t + 1]};
#pragma unroll
          for (int h = 0; h < 2; ++h) dmma_884(d, ColP[(lr0 + g) * SP + 4 * h + t], r1[h]);
          pivot_inverse(kblk + 1, d[0], d[1]);
        }
      } else {
        // S3: R' = D^-1 R outside K, I + D^-1 on K's columns; an 8-column block
        // per warp at a time, two MMAs with D^-1 as the row operand
        if (tile) {
          const double a0 = Dinv[g * SP + t], a1 = Dinv[g * SP + 4 + t];
          for (int cb = warp; cb < CBK; cb += NW) {
            double d[2];
            if (cb == kblk) {
              d[0] = Dinv[g * SP + 2 * t] + ((g == 2 * t) ? 1.0 : 0.0);
              d[1] = Dinv[g * SP + 2 * t + 1] + ((g == 2 * t + 1) ? 1.0 : 0.0);
            } else {
              const double b0 = RowPT[(cb * 8 + g) * SP + t], b1 = RowPT[(cb * 8 + g) * SP + 4 + t];
              d[0] = 0.0;
              d[1] = 0.0;
              dmma_884(d, a0, b0);
              dmma_884(d, a1, b1);
            }
            RowNT[(cb * 8 + 2 * t) * SP + g] = d[0];
            RowNT[(cb * 8 + 2 * t + 1) * SP + g] = d[1];
          }
        }
        __syncthreads();

        if (tile) {
          // S4: W += (-C') R', two MMAs per sub-block
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            double a[WR], b[WC];
#pragma unroll
            for (int i = 0; i < WR; ++i) a[i] = ColP[lrow(i) * SP + 4 * h + t];
#pragma unroll
            for (int j = 0; j < WC; ++j) b[j] = RowNT[((wc + WGC * j) * 8 + g) * SP + 4 * h + t];
#pragma unroll
            for (int i = 0; i < WR; ++i)
#pragma unroll
              for (int j = 0; j < WC; ++j) dmma_884(W[i][j], a[i], b[j]);
          }
        } else if (kblk + 1 < nbe && rank == (kblk + 1) % CL) {
          // the next pivot block, updated exactly as its holders update it, then inverted
          const int lr0 = ((kblk + 1) / CL) * 8;
          const double* Dn = B + S::off_Dnext;
          double d[2] = {Dn[g * SP + 2 * t], Dn[g * SP + 2 * t + 1]};
#pragma unroll
          for (int h = 0; h < 2; ++h)
            dmma_884(d, ColP[(lr0 + g) * SP + 4 * h + t], RowNT[(kb + 8 + g) * SP + 4 * h + t]);
          pivot_inverse(kblk + 1, d[0], d[1]);
        }
      }
    }

    // ---- store N^-1, or B = N^-1 diag(R) with the fused epilogue
    double* __restrict__ Og = bv.out + bv.offA[s];
    if (tile) {
      const double* __restrict__ Rs = ep.R ? ep.R + ep.offv[s] : nullptr;
#pragma unroll
      for (int i = 0; i < WR; ++i) {
        const int r = grow(i);
        if (r < n) {
#pragma unroll
          for (int j = 0; j < WC; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int c = gcol(j, e);
              if (c < n) Og[int64_t(r) * n + c] = Rs ? mul_rn(W[i][j][e], __ldg(Rs + c)) : W[i][j][e];
            }
        }
      }
    }
    if (ep.C) {
      // running totals of each row this CTA holds, from the B just written (L2):
      // a warp takes 32 local rows and walks them in 32 x 32 tiles, loaded and
      // stored coalesced through shared memory (the panel buffers, free now),
      // each lane adding its own row left to right as the reference does.
      // A cluster barrier first: warps of this CTA may still be reading the
      // last step's panels in these buffers.
      cluster_barrier<CL>();
      double* __restrict__ Cg = ep.C + bv.offA[s];
      constexpr int NG = (LP + 31) / 32;
      if (tile && warp < NG) {
        double* tl = sm + warp * (32 * 33);
        auto row_of = [&](int lr) -> int {
          return (lr < LP) ? ((((lr >> 3) * CL) + rank) * 8 + (lr & 7)) : n;
        };
        double total = 0.0;
        for (int c0 = 0; c0 < n; c0 += 32) {
          const int c = c0 + lane;
#pragma unroll 8
          for (int k = 0; k < 32; ++k) {
            const int rk = row_of(warp * 32 + k);
            tl[k * 33 + lane] = (rk < n && c < n) ? __ldcg(Og + int64_t(rk) * n + c) : 0.0;
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
            const int rk = row_of(warp * 32 + k);
            if (rk < n && c < n) Cg[int64_t(rk) * n + c] = tl[k * 33 + lane];
          }
          __syncwarp();
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
