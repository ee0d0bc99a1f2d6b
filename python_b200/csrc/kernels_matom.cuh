// Macro-atom epilogue and consumer on the GPU.
//
// After the jumping matrix N = I - Q/Q_norm of every cell is inverted, the
// reference forms B = N^-1 diag(R) (source/macro_accelerate.c:325-334) and, for
// every macro-atom activation, walks one row of B with a running total until it
// reaches a uniform random number z (matom_deactivation_from_matrix,
// macro_accelerate.c:995-1008).  matom_epilogue_kernel forms B in place of the
// inverse and, optionally, the row running totals C[r][c] = sum_{c'<=c} B[r][c'],
// accumulated left to right exactly as that loop accumulates them, so that a
// draw becomes a search of C.  matom_sample_kernel answers a batch of draws.
#pragma once
#include "ss_common.cuh"

namespace ss {

// The systems an epilogue launch serves: all nsys of the batch, or the listed
// ones (list[0 .. count), the count read from count_dev when that is set: a
// list filled on the device by the certified kernel).
struct EpiList {
  const int* list = nullptr;
  int count = 0;
  const int* count_dev = nullptr;
};
__device__ __forceinline__ int epi_count(int nsys, const EpiList& el) {
  if (!el.list) return nsys;
  return el.count_dev ? *el.count_dev : el.count;
}
__device__ __forceinline__ int epi_system(int i, const EpiList& el) { return el.list ? el.list[i] : i; }

// One CTA per system (grid-stride), one thread per row.  A singular system
// (status != 0) gets B = 0 and C = 0: the reference's output of invert_matrix
// is a zero-filled buffer that the failed call leaves untouched.
__global__ void __launch_bounds__(128) matom_epilogue_kernel(int nsys, const int* __restrict__ n,
                                                             const int64_t* __restrict__ offA,
                                                             const int64_t* __restrict__ offv,
                                                             double* __restrict__ B,
                                                             const double* __restrict__ R,
                                                             double* __restrict__ C,
                                                             const int* __restrict__ status, EpiList el) {
  const int count = epi_count(nsys, el);
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const int s = epi_system(i, el);
    const int ns = n[s];
    const bool ok = status[s] == 0;
    double* __restrict__ Bs = B + offA[s];
    double* __restrict__ Cs = C ? C + offA[s] : nullptr;
    const double* __restrict__ Rs = R + offv[s];
    for (int r = threadIdx.x; r < ns; r += blockDim.x) {
      double* __restrict__ brow = Bs + int64_t(r) * ns;
      double total = 0.0;
      for (int c = 0; c < ns; ++c) {
        const double b = ok ? mul_rn(brow[c], __ldg(Rs + c)) : 0.0;
        brow[c] = b;
        total = add_rn(total, b);
        if (Cs) Cs[int64_t(r) * ns + c] = total;
      }
    }
  }
}

// The same for systems whose n x n block fits the dynamic shared memory: the
// block is scaled with coalesced loads and stores, staged in shared memory,
// and each thread runs its row's running total there (the same additions in
// the same order), after which the totals leave with coalesced stores.
__global__ void __launch_bounds__(128) matom_epilogue_tile_kernel(int nsys, const int* __restrict__ n,
                                                                  const int64_t* __restrict__ offA,
                                                                  const int64_t* __restrict__ offv,
                                                                  double* __restrict__ B,
                                                                  const double* __restrict__ R,
                                                                  double* __restrict__ C,
                                                                  const int* __restrict__ status, EpiList el) {
  extern __shared__ double tile[];   // [n][n] of the current system
  const int count = epi_count(nsys, el);
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const int s = epi_system(i, el);
    const int ns = n[s];
    const int nn = ns * ns;
    const bool ok = status[s] == 0;
    double* __restrict__ Bs = B + offA[s];
    const double* __restrict__ Rs = R + offv[s];
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      const int c = e % ns;
      const double b = ok ? mul_rn(Bs[e], __ldg(Rs + c)) : 0.0;
      Bs[e] = b;
      tile[e] = b;
    }
    if (C) {
      __syncthreads();
      for (int r = threadIdx.x; r < ns; r += blockDim.x) {
        double total = 0.0;
        for (int c = 0; c < ns; ++c) {
          total = add_rn(total, tile[r * ns + c]);
          tile[r * ns + c] = total;
        }
      }
      __syncthreads();
      double* __restrict__ Cs = C + offA[s];
      for (int e = threadIdx.x; e < nn; e += blockDim.x) Cs[e] = tile[e];
    }
    __syncthreads();
  }
}

// Query i draws from row level[i] of system sys[i] with the number z[i]: the
// reference returns 0 when z <= 0 and otherwise the first column whose running
// total is not below z.  target[i] = -1 when the row total stays below z (the
// reference's loop would run past the row), -2 for a system or level out of range.
__global__ void __launch_bounds__(256) matom_sample_kernel(int nq, int nsys, const int* __restrict__ n,
                                                           const int64_t* __restrict__ offA,
                                                           const double* __restrict__ C,
                                                           const int* __restrict__ sys,
                                                           const int* __restrict__ level,
                                                           const double* __restrict__ z,
                                                           int* __restrict__ target) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const int s = sys[i], u = level[i];
  if (s < 0 || s >= nsys) { target[i] = -2; return; }
  const int ns = n[s];
  if (u < 0 || u >= ns) { target[i] = -2; return; }
  const double zz = z[i];
  if (!(0.0 < zz)) { target[i] = 0; return; }
  const double* __restrict__ row = C + offA[s] + int64_t(u) * ns;
  int j = -1;
  for (int c = 0; c < ns; ++c) {
    if (!(__ldg(row + c) < zz)) { j = c; break; }
  }
  target[i] = j;
}

}  // namespace ss
