// GPU assembly of the ion-balance rate matrices (populate_ion_rate_matrix,
// source/matrix_ion.c:444-659) from per-cell coefficient tables.
//
// The reference's matrix is block-diagonal by element once each element's
// first row is replaced by ones (:633-655), so it is assembled straight into
// the per-element systems the batched solve takes.  Every entry of column nn
// comes from ion nn's own coefficients: photoionisation and direct
// ionisation feed the entry below the diagonal, radiative, three-body and
// dielectronic recombination and charge-exchange recombination the entry
// above it, inner-shell ionisation the entries up to ten rows below.  One
// warp assembles one (cell, element) block with a lane per column, each
// entry accumulated in the reference's block order with one rounding per
// product and per sum (no contraction), so the blocks are bit-identical to
// the reference's.
#pragma once
#include "ss_common.cuh"

namespace ss {

struct IonAsmView {
  int nions, nelem, ncx, n_inner;
  const int* elem_first;   // [nelem]
  const int* elem_n;       // [nelem]
  const int64_t* blk_off;  // [nelem] offset of element e's block inside a cell's blocks
  int64_t blk_cell;        // doubles of one cell's blocks
  const int* ion_z;        // [nions] atomic number
  const int* ion_istate;   // [nions] stage, 1 = neutral
  const int* ion_flags;    // [nions] bit 0: highest stage, bit 1: DI data, bit 2: DR data
  const int* cx_start;     // [nions + 1] charge-exchange ionisation entries of each ion (hydrogen partner)
  const int* cx_idx;       // entry indices, ascending
  const int* in_start;     // [nions + 1] inner-shell rates of each ion with yield data
  const int* in_idx;       // rate indices, ascending
  const int* in_yield;     // their yield rows
  const double* yield;     // [n_yield][10]
  const double *pi, *rr, *di, *qr, *dr, *cxr;   // [ncell][nions]
  const double* cxi;       // [ncell][ncx]
  const double* inner;     // [ncell][n_inner]
  int count;               // cells to assemble
  const int* cells;        // [count] cell index of each item
  const double *ne, *nh1, *nh2;   // [count]
  double* A;               // [count][blk_cell]
  double* b;               // [count][nions]
};

constexpr int kIonAsmThreads = 128;

__global__ void __launch_bounds__(kIonAsmThreads) ion_assemble_kernel(IonAsmView v) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t(blockIdx.x) * kIonAsmThreads + threadIdx.x) >> 5;
  if (w >= int64_t(v.count) * v.nelem) return;
  const int item = int(w / v.nelem), e = int(w - int64_t(item) * v.nelem);
  const int cell = v.cells[item];
  const int ne_ = v.elem_n[e], f = v.elem_first[e];
  const double xne = v.ne[item], nh1 = v.nh1[item], nh2 = v.nh2[item];
  double* __restrict__ blk = v.A + int64_t(item) * v.blk_cell + v.blk_off[e];
  const int64_t rc = int64_t(cell) * v.nions;
  for (int r = lane; r < ne_; r += 32) v.b[int64_t(item) * v.nions + f + r] = (r == 0) ? 1.0 : 0.0;

  for (int cg = 0; cg < ne_; cg += 32) {
    const int cl = cg + lane;
    const bool live = cl < ne_;
    // every row of the column: the element's first row is all ones, the rest zero
    if (live)
      for (int r = 0; r < ne_; ++r) blk[int64_t(r) * ne_ + cl] = (r == 0) ? 1.0 : 0.0;
    if (!live) continue;
    const int nn = f + cl;
    const int flags = v.ion_flags[nn];
    const bool top = flags & 1, has_di = flags & 2, has_dr = flags & 4;
    const bool below = cl + 1 < ne_;   // ion nn + 1 is of the same element
    double diag = 0.0, sub = 0.0, sup = 0.0;
    double inn[9];
#pragma unroll
    for (int d = 0; d < 9; ++d) inn[d] = 0.0;
    // photoionisation (:477-497)
    if (!top) diag = sub_rn(diag, v.pi[rc + nn]);
    if (!top && below) sub = add_rn(sub, v.pi[rc + nn]);
    // direct ionisation (:501-520)
    if (!top && has_di) diag = sub_rn(diag, mul_rn(xne, v.di[rc + nn]));
    if (!top && below && has_di) sub = add_rn(sub, mul_rn(xne, v.di[rc + nn]));
    // radiative and three-body recombination (:525-544)
    if (cl != 0) {
      const double t = mul_rn(xne, add_rn(v.rr[rc + nn], mul_rn(xne, v.qr[rc + nn])));
      diag = sub_rn(diag, t);
      sup = add_rn(sup, t);
    }
    // dielectronic recombination (:548-572); the populating term takes the
    // flag of the lower ion
    if (cl != 0 && has_dr) diag = sub_rn(diag, mul_rn(xne, v.dr[rc + nn]));
    if (cl != 0 && (v.ion_flags[nn - 1] & 4)) sup = add_rn(sup, mul_rn(xne, v.dr[rc + nn]));
    // charge-exchange recombination (:576-586); the term above a neutral ion
    // falls outside the block and is zero (checked on the host)
    if (v.ncx > 0 && v.ion_z[nn] != 1 && v.ion_istate[nn] != 0) {
      const double t = mul_rn(v.cxr[rc + nn], nh1);
      diag = sub_rn(diag, t);
      if (cl != 0) sup = add_rn(sup, t);
    }
    // charge-exchange ionisation against hydrogen (:590-596), entries in order
    for (int k = v.cx_start[nn]; k < v.cx_start[nn + 1]; ++k) {
      const double t = mul_rn(v.cxi[int64_t(cell) * v.ncx + v.cx_idx[k]], nh2);
      diag = sub_rn(diag, t);
      sub = add_rn(sub, t);
    }
    // inner-shell ionisation with electron yields (:599-613), rates in order
    const int nel = min(v.ion_z[nn] - v.ion_istate[nn] + 1, 11);
    for (int k = v.in_start[nn]; k < v.in_start[nn + 1]; ++k) {
      const double rate = v.inner[int64_t(cell) * v.n_inner + v.in_idx[k]];
      const double* __restrict__ prob = v.yield + int64_t(v.in_yield[k]) * 10;
      diag = sub_rn(diag, rate);
      if (nel > 1) sub = add_rn(sub, mul_rn(rate, prob[0]));
#pragma unroll
      for (int d = 2; d <= 10; ++d)
        if (d < nel) inn[d - 2] = add_rn(inn[d - 2], mul_rn(rate, prob[d - 1]));
    }
    // the structured entries over the zeros, in this lane's program order
    if (cl != 0) blk[int64_t(cl) * ne_ + cl] = diag;
    if (below) blk[int64_t(cl + 1) * ne_ + cl] = sub;
    if (cl >= 2) blk[int64_t(cl - 1) * ne_ + cl] = sup;
#pragma unroll
    for (int d = 2; d <= 10; ++d)
      if (cl + d < ne_) blk[int64_t(cl + d) * ne_ + cl] = inn[d - 2];
  }
}

}  // namespace ss
