// Tuning library of the certified Gauss-Jordan classes (kernels_cert.cuh).
//
// Not part of the engine: python_b200/autotune.py (--family cgj) compiles this
// file once per padded order P, with SS_TUNE_CGJ_LIST naming a file of the
// SS_TUNE_CGJ(P, WGR, WGC, CL, MINB, ST) candidates of that order (taken from
// tune_cgj_candidates.inc), times each candidate on device-resident batches
// and writes cgj_classes.inc, which the engine build compiles in.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels_cert.cuh"

#ifndef SS_TUNE_CGJ_LIST
#error "SS_TUNE_CGJ_LIST names the candidate list of one padded order"
#endif

namespace {

struct Candidate {
  int P, WGR, WGC, CL, MINB, ST;
  const void* fn;
  int threads;
  size_t smem;
};

#define SS_TUNE_CGJ(P, WGR, WGC, CL, MINB, ST)                                                     \
  {P, WGR, WGC, CL, MINB, ST ? 1 : 0,                                                            \
   reinterpret_cast<const void*>(&ss::cgj_inverse_kernel<P, WGR, WGC, CL, MINB, ST>),           \
   ss::CgjShape<P, WGR, WGC, CL, MINB, ST>::NTH, ss::CgjShape<P, WGR, WGC, CL, MINB, ST>::dyn_smem},
const Candidate kCand[] = {
#include SS_TUNE_CGJ_LIST
};
#undef SS_TUNE_CGJ
constexpr int kNumCand = int(sizeof(kCand) / sizeof(kCand[0]));

}  // namespace

extern "C" {

int sirocco_tune_count(void) { return kNumCand; }

// Configuration of candidate i: P, WGR, WGC, CL, CTAs per SM asked, staged.
int sirocco_tune_info(int i, int* cfg) {
  if (i < 0 || i >= kNumCand) return -1;
  const Candidate& c = kCand[i];
  cfg[0] = c.P; cfg[1] = c.WGR; cfg[2] = c.WGC; cfg[3] = c.CL; cfg[4] = c.MINB; cfg[5] = c.ST;
  return 0;
}

// Inverts the nsys matrices of the device batch (orders <= P of candidate i,
// layout arrays on the device; every matrix must pass the certificate) reps
// times with candidate i and returns the fastest launch in *ms; *resident gets
// the CTAs per SM the configuration runs.  d_scratch holds 4 * nsys + 4 ints
// for the fallback lists the kernel would fill.
int sirocco_tune_time(int i, int nsys, const int* d_n, const int64_t* d_offA, const double* d_A, double* d_out,
                      int* d_status, const int* d_list, int* d_scratch, int reps, float* ms, int* resident) {
  if (i < 0 || i >= kNumCand || nsys < 1 || reps < 1) return -1;
  const Candidate& c = kCand[i];
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(c.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(c.smem)))) return int(e);
  int dev = 0, sms = 0;
  if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return int(e);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = unsigned(c.CL);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(unsigned(c.threads));
  cfg.dynamicSmemBytes = c.smem;
  cfg.attrs = at;
  cfg.numAttrs = c.CL > 1 ? 1 : 0;
  int slots = 0;   // matrices in flight (clusters, or CTAs)
  if (c.CL > 1) {
    cfg.gridDim = dim3(unsigned(c.CL * sms));
    if ((e = cudaOccupancyMaxActiveClusters(&slots, c.fn, &cfg))) return int(e);
  } else {
    int nb = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, c.fn, c.threads, c.smem))) return int(e);
    slots = nb * sms;
  }
  if (slots < 1) return -2;
  const int grid = (nsys < slots ? nsys : slots) * c.CL;
  cfg.gridDim = dim3(unsigned(grid));
  int* xcls = d_scratch;                  // [nsys] all zero: one fallback list
  int* fboff = d_scratch + nsys;          // [2]
  int* fbcount = d_scratch + nsys + 2;    // [1]
  int* fblist = d_scratch + nsys + 4;     // [nsys]
  if ((e = cudaMemset(d_scratch, 0, sizeof(int) * size_t(nsys + 4)))) return int(e);
  ss::BatchView bv{};
  bv.n = d_n;
  bv.offA = d_offA;
  bv.A = d_A;
  bv.out = d_out;
  bv.status = d_status;
  bv.list = d_list;
  bv.count = nsys;
  ss::CertArgs ca{xcls, fboff, fblist, fbcount};
  ss::CertEpi ep{};
  void* args[] = {&bv, &ca, &ep};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int rc = 0;
  for (int r = 0; r <= reps && rc == 0; ++r) {   // launch 0 warms up
    cudaEventRecord(e0);
    if ((e = cudaLaunchKernelExC(&cfg, c.fn, args))) rc = int(e);
    cudaEventRecord(e1);
    if (!rc && (e = cudaEventSynchronize(e1))) rc = int(e);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (r > 0 && t < best) best = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  *resident = slots * c.CL / sms;
  return rc;
}

}  // extern "C"
