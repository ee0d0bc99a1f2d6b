// GPU assembly of the macro-atom jump matrices (the Q / R assembly and
// normalisation of calc_matom_matrix, source/macro_accelerate.c:82-284).
//
// Row u of Q, R and the normalisation Q_norm come only from level u's own
// jumps (the k-packet row from the macro lines' and continua's cooling
// rates), so one thread builds one row: it zeroes its row, accumulates every
// jump's contributions in the reference's order with one rounding per
// product, sum and difference, and then forms N = I - Q / Q_norm and
// R / Q_norm.  The rows of a block are built in shared memory when they fit
// (every += stays on chip) and leave with one coalesced copy: consecutive
// threads own consecutive rows of N.  Larger models build them in place.
#pragma once
#include "ss_common.cuh"

namespace ss {

struct MatomAsmView {
  int nlev, n_bbd, n_aug, n_bfd, n_bbu, n_bfu, n_kbb, n_kbf;
  const double* ex;         // [nlev]
  const double* aug_rate;   // [n_aug]
  const int *bbd_start, *bbd_t, *aug_start, *aug_t, *bfd_start, *bfd_t, *bbu_start, *bbu_t, *bfu_start, *bfu_t;
  const int *kbb_t, *kbf_t;
  // per cell: [ncell][n_x] per jump list, [ncell] for kr and ne
  const double *bbd_rad, *bbd_coll, *bfd_sp, *bfd_qrec, *bbu_rad, *bbu_coll;
  const double *bfu_gamma, *bfu_alpha, *bfu_ratio, *bfu_qion, *kbb, *kbf, *kr, *ne;
  int ncell;
  double* N;   // [ncell][nlev + 1][nlev + 1]
  double* R;   // [ncell][nlev + 1]
};

// Row u of cell `cell` into q (zeroed): Q, then N = I - Q / Q_norm; R / Q_norm
// to v.R.
__device__ __forceinline__ void assemble_row(const MatomAsmView& v, int cell, int u, int nr, int K,
                                             double* __restrict__ q) {
  double r = 0.0, qn = 0.0;
  const double ne = v.ne[cell];
  if (u < K) {
    const double eu = v.ex[u];
    // bound-bound down (:98-123)
    for (int j = v.bbd_start[u]; j < v.bbd_start[u + 1]; ++j) {
      const double rad = v.bbd_rad[int64_t(cell) * v.n_bbd + j], coll = v.bbd_coll[int64_t(cell) * v.n_bbd + j];
      const int t = v.bbd_t[j];
      const double de = sub_rn(eu, v.ex[t]);
      const double qc = mul_rn(add_rn(rad, mul_rn(coll, ne)), v.ex[t]);
      q[t] = add_rn(q[t], qc);
      const double qk = mul_rn(mul_rn(coll, ne), de);
      q[K] = add_rn(q[K], qk);
      const double rc = mul_rn(rad, de);
      r = add_rn(r, rc);
      qn = add_rn(qn, add_rn(add_rn(qc, qk), rc));
    }
    // Auger (:126-145)
    for (int j = v.aug_start[u]; j < v.aug_start[u + 1]; ++j) {
      const double rate = v.aug_rate[j];
      const int t = v.aug_t[j];
      const double qc = mul_rn(rate, v.ex[t]);
      q[t] = add_rn(q[t], qc);
      const double qk = mul_rn(rate, sub_rn(eu, v.ex[t]));
      q[K] = add_rn(q[K], qk);
      qn = add_rn(qn, add_rn(qc, qk));
    }
    // bound-free down (:148-174), only for a positive rate
    for (int j = v.bfd_start[u]; j < v.bfd_start[u + 1]; ++j) {
      const double sp = v.bfd_sp[int64_t(cell) * v.n_bfd + j], qr = v.bfd_qrec[int64_t(cell) * v.n_bfd + j];
      const double bf = mul_rn(add_rn(sp, mul_rn(qr, ne)), ne);
      const int t = v.bfd_t[j];
      if (bf > 0.0) {
        const double de = sub_rn(eu, v.ex[t]);
        const double qc = mul_rn(bf, v.ex[t]);
        q[t] = add_rn(q[t], qc);
        const double qk = mul_rn(mul_rn(mul_rn(qr, ne), ne), de);
        q[K] = add_rn(q[K], qk);
        const double rc = mul_rn(mul_rn(ne, sp), de);
        r = add_rn(r, rc);
        qn = add_rn(qn, add_rn(add_rn(qc, qk), rc));
      }
    }
    // bound-bound up (:179-191)
    for (int j = v.bbu_start[u]; j < v.bbu_start[u + 1]; ++j) {
      const double rad = v.bbu_rad[int64_t(cell) * v.n_bbu + j], coll = v.bbu_coll[int64_t(cell) * v.n_bbu + j];
      const int t = v.bbu_t[j];
      const double qc = mul_rn(add_rn(rad, mul_rn(coll, ne)), eu);
      q[t] = add_rn(q[t], qc);
      qn = add_rn(qn, qc);
    }
    // bound-free up (:194-222): a negative rate counts as zero
    for (int j = v.bfu_start[u]; j < v.bfu_start[u + 1]; ++j) {
      const int64_t k = int64_t(cell) * v.n_bfu + j;
      const int t = v.bfu_t[j];
      double qc = mul_rn(add_rn(sub_rn(v.bfu_gamma[k], mul_rn(mul_rn(v.bfu_alpha[k], ne), v.bfu_ratio[k])),
                                mul_rn(v.bfu_qion[k], ne)),
                         eu);
      if (qc < 0.0) qc = 0.0;
      q[t] = add_rn(q[t], qc);
      qn = add_rn(qn, qc);
    }
  } else {
    // the k-packet row (:236-263): macro lines, then macro continua, then the
    // k-packet to r-packet channel
    for (int j = 0; j < v.n_kbb; ++j) {
      const double qc = v.kbb[int64_t(cell) * v.n_kbb + j];
      q[v.kbb_t[j]] = add_rn(q[v.kbb_t[j]], qc);
      qn = add_rn(qn, qc);
    }
    for (int j = 0; j < v.n_kbf; ++j) {
      const double qc = v.kbf[int64_t(cell) * v.n_kbf + j];
      q[v.kbf_t[j]] = add_rn(q[v.kbf_t[j]], qc);
      qn = add_rn(qn, qc);
    }
    const double kr = v.kr[cell];
    r = add_rn(r, kr);
    qn = add_rn(qn, kr);
  }
  // N = I - Q / Q_norm, R / Q_norm (:270-284)
  if (qn > 0.0)
    for (int t = 0; t < nr; ++t) q[t] = div_rn(-q[t], qn);
  q[u] = 1.0;
  v.R[int64_t(cell) * nr + u] = (qn > 0.0) ? div_rn(r, qn) : r;
}

constexpr int kMatomAsmThreads = 128;

// staged: the block's rows live in dynamic shared memory ([blockDim][nlev + 1])
__global__ void __launch_bounds__(kMatomAsmThreads) matom_assemble_kernel(MatomAsmView v, bool staged) {
  extern __shared__ double srow[];
  const int nr = v.nlev + 1, K = v.nlev;
  const int64_t nrows = int64_t(v.ncell) * nr;
  const int64_t row0 = int64_t(blockIdx.x) * blockDim.x;
  const int64_t tid = row0 + threadIdx.x;
  if (tid < nrows) {
    const int cell = int(tid / nr), u = int(tid - int64_t(cell) * nr);
    double* __restrict__ q = staged ? srow + int64_t(threadIdx.x) * nr : v.N + tid * nr;
    for (int t = 0; t < nr; ++t) q[t] = 0.0;
    assemble_row(v, cell, u, nr, K, q);
  }
  if (staged) {
    __syncthreads();
    const int64_t nb = min(int64_t(blockDim.x), nrows - row0) * nr;
    double* __restrict__ dst = v.N + row0 * nr;
    for (int64_t e = threadIdx.x; e < nb; e += blockDim.x) dst[e] = srow[e];
  }
}

}  // namespace ss
