// Tuning library of the small-system family (python_b200/_build/libsirocco_tune_small.so).
//
// Not part of the engine: python_b200/autotune.py (--family small) loads it to
// time every candidate of tune_small_candidates.inc on device-resident batches
// of solves, keeps the fastest lane count per padded order and writes
// small_classes.inc, which the engine build compiles in.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels_small.cuh"

namespace {

struct Candidate {
  int NP, G;
  const void* fn;
};

#define SS_TUNE_SMALL(NP, G) {NP, G, reinterpret_cast<const void*>(&ss::small_exact_kernel<ss::kSolve, NP, G>)},
const Candidate kCand[] = {
#include "tune_small_candidates.inc"
};
#undef SS_TUNE_SMALL
constexpr int kNumCand = int(sizeof(kCand) / sizeof(kCand[0]));

}  // namespace

extern "C" {

int sirocco_tune_count(void) { return kNumCand; }

// Configuration of candidate i: NP, G.
int sirocco_tune_info(int i, int* cfg) {
  if (i < 0 || i >= kNumCand) return -1;
  cfg[0] = kCand[i].NP;
  cfg[1] = kCand[i].G;
  return 0;
}

// Solves the nsys systems of the device batch (orders <= NP of candidate i,
// layout arrays on the device) reps times with candidate i and returns the
// fastest launch in *ms; *resident gets the CTAs per SM the configuration runs.
int sirocco_tune_time(int i, int nsys, const int* d_n, const int64_t* d_offA, const int64_t* d_offv,
                      const double* d_A, const double* d_b, double* d_x, int* d_status, const int* d_list, int reps,
                      float* ms, int* resident) {
  if (i < 0 || i >= kNumCand || nsys < 1 || reps < 1) return -1;
  const Candidate& c = kCand[i];
  cudaError_t e;
  int nb = 0, dev = 0, sms = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, c.fn, ss::kSmallThreads, 0))) return int(e);
  if (nb < 1) return -2;
  if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return int(e);
  const int per_block = ss::kSmallThreads / c.G;
  const int need = (nsys + per_block - 1) / per_block;
  const int grid = need < nb * sms ? need : nb * sms;
  ss::BatchView bv{};
  bv.n = d_n;
  bv.offA = d_offA;
  bv.offv = d_offv;
  bv.A = d_A;
  bv.b = d_b;
  bv.out = d_x;
  bv.status = d_status;
  bv.list = d_list;
  bv.count = nsys;
  void* args[] = {&bv};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int rc = 0;
  for (int r = 0; r <= reps && rc == 0; ++r) {   // launch 0 warms up
    cudaEventRecord(e0);
    if ((e = cudaLaunchKernel(c.fn, dim3(grid), dim3(ss::kSmallThreads), args, 0, 0))) rc = int(e);
    cudaEventRecord(e1);
    if (!rc && (e = cudaEventSynchronize(e1))) rc = int(e);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (r > 0 && t < best) best = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  *resident = nb;
  return rc;
}

}  // extern "C"
