// Tuning library of the CTA kernel family (python_b200/libsirocco_tune.so).
//
// Not part of the engine: python_b200/autotune.py loads it to time every
// candidate configuration of tune_candidates.inc on device-resident batches,
// keeps the fastest per padded order and writes cta_classes.inc, which the
// engine build compiles in.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels_cta.cuh"

namespace {

struct Candidate {
  int P, NT, RG, CC, PW, GM, MINB;
  const void* fn;
  size_t smem;
  int64_t slab;
};

#define SS_TUNE(P, NT, RG, CC, PW, GM, MINB)                                                          \
  {P, NT, RG, CC, PW, GM ? 1 : 0, MINB,                                                               \
   reinterpret_cast<const void*>(&ss::cta_exact_kernel<ss::kInvert, P, NT, RG, CC, PW, GM, MINB>),    \
   ss::CtaShape<ss::kInvert, P, NT, RG, CC, PW, GM, MINB>::dyn_smem,                                 \
   ss::CtaShape<ss::kInvert, P, NT, RG, CC, PW, GM, MINB>::slab},
const Candidate kCand[] = {
#include "tune_candidates.inc"
};
#undef SS_TUNE
constexpr int kNumCand = int(sizeof(kCand) / sizeof(kCand[0]));

}  // namespace

extern "C" {

int sirocco_tune_count(void) { return kNumCand; }

// Configuration of candidate i: P, threads, RG, CC, panel warps, global memory, CTAs per SM asked.
int sirocco_tune_info(int i, int* cfg) {
  if (i < 0 || i >= kNumCand) return -1;
  const Candidate& c = kCand[i];
  cfg[0] = c.P; cfg[1] = c.NT; cfg[2] = c.RG; cfg[3] = c.CC; cfg[4] = c.PW; cfg[5] = c.GM; cfg[6] = c.MINB;
  return 0;
}

// Inverts the nsys systems of the device batch (orders <= P of candidate i,
// layout arrays on the device) reps times with candidate i and returns the
// fastest launch in *ms; *resident gets the CTAs per SM the configuration runs.
int sirocco_tune_time(int i, int nsys, const int* d_n, const int64_t* d_offA, const double* d_A, double* d_out,
                      int* d_status, const int* d_list, int reps, float* ms, int* resident) {
  if (i < 0 || i >= kNumCand || nsys < 1 || reps < 1) return -1;
  const Candidate& c = kCand[i];
  cudaError_t e;
  if (c.smem > 0 && (e = cudaFuncSetAttribute(c.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(c.smem))))
    return int(e);
  int nb = 0, dev = 0, sms = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, c.fn, c.NT, c.smem))) return int(e);
  if (nb < 1) return -2;
  if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return int(e);
  const int grid = nsys < nb * sms ? nsys : nb * sms;
  double* work = nullptr;
  if (c.slab > 0 && (e = cudaMalloc(&work, sizeof(double) * size_t(c.slab) * grid))) return int(e);
  ss::BatchView bv{d_n, d_offA, nullptr, d_A, nullptr, d_out, d_status, nullptr, d_list, nsys};
  void* args[] = {&bv, &work};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int rc = 0;
  for (int r = 0; r <= reps && rc == 0; ++r) {   // launch 0 warms up
    cudaEventRecord(e0);
    if ((e = cudaLaunchKernel(c.fn, dim3(grid), dim3(c.NT), args, c.smem, 0))) rc = int(e);
    cudaEventRecord(e1);
    if (!rc && (e = cudaEventSynchronize(e1))) rc = int(e);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (r > 0 && t < best) best = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (work) cudaFree(work);
  *ms = best;
  *resident = nb;
  return rc;
}

}  // extern "C"
