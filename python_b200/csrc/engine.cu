// Host runtime and C ABI of the batched dense-solve engine.
//
// A plan groups the systems of one batch layout into size buckets, each served
// by one kernel family (kernels_small.cuh for n <= 32, kernels_cta.cuh for
// n <= 1024; kernels_cert.cuh for the certified inverses of SIROCCO_FAST mode),
// keeps the layout on the device, and launches the buckets on forked streams so
// small and large systems overlap.  A plan with certified buckets runs in two
// phases: the certified kernels first, which append every system that fails
// the certificate to a device-side list per exact size class, then the
// GSL-exact kernels over those lists.
// The drop-in entry points (solve_matrix, invert_matrix) and the host-pointer
// batched calls run through a per-thread context that caches plans and
// grow-only device staging buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <functional>
#include <unordered_map>
#include <vector>

#include "../../include/sirocco_solve.h"
#include "kernels_cert.cuh"
#include "kernels_certl.cuh"
#include "kernels_cta.cuh"
#include "kernels_global.cuh"
#include "kernels_ionasm.cuh"
#include "kernels_matom.cuh"
#include "kernels_matomasm.cuh"
#include "kernels_mixed.cuh"
#include "kernels_small.cuh"

namespace ss {

// ------------------------------------------------------------------ errors --
static thread_local std::string g_last_error;

static void set_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

#define SS_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      set_error("CUDA error %d (%s) at %s:%d", int(e_), cudaGetErrorString(e_), __FILE__, __LINE__); \
      return int(e_);                                                                       \
    }                                                                                       \
  } while (0)

// ---------------------------------------------------------------- kernels --
enum Family : int { kFamSmall = 0, kFamCta = 1, kFamGlobal = 2, kFamCgj = 3, kFamCgjL = 4 };

struct KernelSpec {
  const void* fn = nullptr;
  int threads = 0;
  size_t dyn_smem = 0;
  int sys_per_block = 1;
  int blocks_per_sm = 1;
  int64_t work_slab = 0;   // CTA family with the matrix in global memory: doubles per CTA
  int cluster = 1;         // CTAs per system (certified family above order 128)
  int max_ctas = 0;        // CTAs resident on the whole GPU at once
};

// size classes of the small family (padded row length NP; small_classes.inc,
// chosen by python_b200/autotune.py --family small)
static const int kSmallNP[] = {
#define SS_SMALL_CLASS(I, NP, G) NP,
#include "small_classes.inc"
#undef SS_SMALL_CLASS
};
constexpr int kSmallClasses = int(sizeof(kSmallNP) / sizeof(kSmallNP[0]));
// padded orders of the CTA classes (cta_classes.inc, chosen by python_b200/autotune.py)
static const int kCtaP[] = {
#define SS_CTA_CLASS(I, P, NT, RG, CC, PW, GM, MINB) P,
#include "cta_classes.inc"
#undef SS_CTA_CLASS
};
constexpr int kCtaClasses = int(sizeof(kCtaP) / sizeof(kCtaP[0]));

// padded orders of the certified Gauss-Jordan classes (cgj_classes.inc)
static const int kCgjP[] = {
#define SS_CGJ_CLASS(I, P, WGR, WGC, CL, MINB, ST) P,
#include "cgj_classes.inc"
#undef SS_CGJ_CLASS
};
constexpr int kCgjClasses = int(sizeof(kCgjP) / sizeof(kCgjP[0]));
// below this order the warp-group kernels of the exact path are faster
constexpr int kCgjMinN = 33;
// above the largest register-resident class, certified inverses stream
// through global memory (kernels_certl.cuh): row tiles per pass, CTAs per SM
constexpr int kCgjlRT = 1, kCgjlMinB = 3;

static int small_class(int n) {
  for (int i = 0; i < kSmallClasses; ++i)
    if (n <= kSmallNP[i]) return i;
  return -1;
}
static int cta_class(int n) {
  for (int i = 0; i < kCtaClasses; ++i)
    if (n <= kCtaP[i]) return i;
  return -1;
}
static int cgj_class(int n) {
  if (n < kCgjMinN) return -1;
  for (int i = 0; i < kCgjClasses; ++i)
    if (n <= kCgjP[i]) return i;
  return -1;
}

template <int KIND>
static KernelSpec small_spec(int cls, int mode) {
  KernelSpec k;
  k.threads = kSmallThreads;
#define SS_SMALL_CLASS(I, NP, G)                                                        \
  case I:                                                                               \
    k.fn = (mode == SIROCCO_MIXED && KIND == kSolve)                                    \
               ? reinterpret_cast<const void*>(&small_mixed_solve_kernel<NP, G>)        \
               : reinterpret_cast<const void*>(&small_exact_kernel<KIND, NP, G>);       \
    k.sys_per_block = kSmallThreads / G;                                                \
    break;
  switch (cls) {
#include "small_classes.inc"
    default: break;
  }
#undef SS_SMALL_CLASS
  return k;
}

template <int KIND>
static KernelSpec cta_spec(int cls) {
  KernelSpec k;
#define SS_CTA_CLASS(I, P, NT, RG, CC, PW, GM, MINB)                                    \
  case I: {                                                                             \
    using Sh = CtaShape<KIND, P, NT, RG, CC, PW, GM, MINB>;                             \
    k.fn = reinterpret_cast<const void*>(&cta_exact_kernel<KIND, P, NT, RG, CC, PW, GM, MINB>); \
    k.threads = NT;                                                                     \
    k.dyn_smem = Sh::dyn_smem;                                                          \
    k.work_slab = Sh::slab;                                                             \
    break;                                                                              \
  }
  // the class table, measured per class by python_b200/autotune.py: shared
  // memory for the smallest orders, a global workspace slab above them, where
  // more CTAs per SM (more pivot chains in flight) beat the faster memory
  switch (cls) {
#include "cta_classes.inc"
    default: break;
  }
#undef SS_CTA_CLASS
  return k;
}

static KernelSpec cgj_spec(int cls) {
  KernelSpec k;
#define SS_CGJ_CLASS(I, P, WGR, WGC, CL, MINB, ST)                                      \
  case I: {                                                                              \
    using Sh = CgjShape<P, WGR, WGC, CL, MINB, ST>;                                      \
    k.fn = reinterpret_cast<const void*>(&cgj_inverse_kernel<P, WGR, WGC, CL, MINB, ST>); \
    k.threads = Sh::NTH;                                                             \
    k.dyn_smem = Sh::dyn_smem;                                                       \
    k.cluster = CL;                                                                  \
    break;                                                                           \
  }
  switch (cls) {
#include "cgj_classes.inc"
    default: break;
  }
#undef SS_CGJ_CLASS
  return k;
}

static KernelSpec cgjl_spec() {
  using Sh = CgjlShape<kCgjlRT, kCgjlMinB>;
  KernelSpec k;
  k.fn = reinterpret_cast<const void*>(&cgjl_inverse_kernel<kCgjlRT, kCgjlMinB>);
  k.threads = Sh::NTH;
  k.dyn_smem = Sh::dyn_smem;
  return k;
}

template <int KIND>
static KernelSpec global_spec(int nmax) {
  KernelSpec k;
  k.fn = (global_panel_width(nmax) == 16) ? reinterpret_cast<const void*>(&global_exact_kernel<KIND, 16>)
                                          : reinterpret_cast<const void*>(&global_exact_kernel<KIND, 8>);
  k.threads = kGThreads;
  k.dyn_smem = global_smem_bytes(nmax);
  return k;
}

static int finish_spec(KernelSpec& k) {
  if (!k.fn) {
    set_error("no kernel for this size class");
    return SIROCCO_ESIZE;
  }
  if (k.dyn_smem > 0)
    SS_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(k.dyn_smem)));
  int nb = 0;
  SS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k.fn, k.threads, k.dyn_smem));
  if (nb < 1) {
    set_error("kernel does not fit on an SM (threads %d, shared %zu)", k.threads, k.dyn_smem);
    return SIROCCO_ESIZE;
  }
  k.blocks_per_sm = nb;
  int dev = 0, sms = 0;
  SS_CUDA(cudaGetDevice(&dev));
  SS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  k.max_ctas = nb * sms;
  if (k.cluster > 1) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = unsigned(k.cluster);
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(unsigned(k.cluster * sms));
    cfg.blockDim = dim3(unsigned(k.threads));
    cfg.dynamicSmemBytes = k.dyn_smem;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl = 0;
    SS_CUDA(cudaOccupancyMaxActiveClusters(&ncl, k.fn, &cfg));
    if (ncl < 1) {
      set_error("a cluster of %d CTAs (threads %d, shared %zu) cannot be scheduled", k.cluster, k.threads,
                k.dyn_smem);
      return SIROCCO_ESIZE;
    }
    k.max_ctas = ncl * k.cluster;
  }
  return 0;
}

// ------------------------------------------------------------------- plans --
struct Bucket {
  Family fam;
  int cls;        // size class (small / cta) or nmax (global)
  int count;
  int list_off;
  KernelSpec spec;
  int grid;
  int64_t slab;   // scratch elements per CTA (global solves, CTA classes in global memory)
  int64_t scratch_off;
  int phase;      // 1: certified kernels and directly listed systems; 2: fallback lists
  int fb;         // phase 2: index of the fallback list this launch serves
  int q;          // streamed certified inverses: index of the launch's queue counter
};

}  // namespace ss

struct sirocco_plan {
  int kind = 0;
  int mode = 0;
  int nsys = 0;
  int device = 0;
  int num_sms = 0;
  int64_t totA = 0, totV = 0;
  std::vector<ss::Bucket> buckets;
  int* d_n = nullptr;
  int64_t* d_offA = nullptr;
  int64_t* d_offv = nullptr;
  int* d_list = nullptr;
  double* d_scratch = nullptr;
  int64_t scratch_elems = 0;   // workspace doubles the buckets need
  bool own_scratch = true;     // false: d_scratch points into a pipeline's shared workspace
  // certified inverses: per system, the fallback list of its exact size class
  int nfb = 0;                 // fallback lists (exact classes that certified systems belong to)
  int nq = 0;                  // queue counters (after the fallback counts in d_fbcount)
  std::vector<int> fb_off;     // start of each list in d_fblist
  int* d_xcls = nullptr;
  int* d_fboff = nullptr;
  int* d_fblist = nullptr;
  int* d_fbcount = nullptr;
  ss::CertEpi epi;             // set only around a matom_matrices_batched run
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev;
  cudaEvent_t ev_fork = nullptr;
};

namespace ss {

static void plan_free(sirocco_plan* p) {
  if (!p) return;
  cudaFree(p->d_n);
  cudaFree(p->d_offA);
  cudaFree(p->d_offv);
  cudaFree(p->d_list);
  cudaFree(p->d_xcls);
  cudaFree(p->d_fboff);
  cudaFree(p->d_fblist);
  cudaFree(p->d_fbcount);
  if (p->own_scratch) cudaFree(p->d_scratch);
  for (auto s : p->side) cudaStreamDestroy(s);
  for (auto e : p->ev) cudaEventDestroy(e);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  delete p;
}

// Host-side check of a batch layout, before anything touches the device: every
// order in 1..SIROCCO_MAX_N, every offset non-negative, and no two systems'
// output ranges overlapping (the inverse of system s is written at offA[s], a
// solution at offv[s]; matrices of a solve are only read and may share
// storage).  Packed layouts, whose offsets increase, are checked in one pass;
// others are sorted first.
static int check_layout(int kind, int nsys, const int* n, const int64_t* offA, const int64_t* offv) {
  if (nsys < 0 || (nsys > 0 && (!n || !offA || (kind == kSolve && !offv)))) {
    set_error("invalid layout arguments");
    return SIROCCO_EINVAL;
  }
  for (int s = 0; s < nsys; ++s) {
    if (n[s] < 1 || n[s] > SIROCCO_MAX_N) {
      set_error("system %d has order %d (supported 1..%d)", s, n[s], SIROCCO_MAX_N);
      return n[s] < 1 ? SIROCCO_EINVAL : SIROCCO_ESIZE;
    }
    if (offA[s] < 0 || (kind == kSolve && offv[s] < 0)) {
      set_error("system %d has a negative offset", s);
      return SIROCCO_EINVAL;
    }
  }
  const int64_t* off = (kind == kSolve) ? offv : offA;
  auto len = [&](int s) { return (kind == kSolve) ? int64_t(n[s]) : int64_t(n[s]) * n[s]; };
  bool sorted = true;
  for (int s = 0; s + 1 < nsys && sorted; ++s) sorted = off[s] <= off[s + 1];
  std::vector<int> order;
  if (!sorted) {
    order.resize(nsys);
    for (int s = 0; s < nsys; ++s) order[s] = s;
    std::sort(order.begin(), order.end(), [&](int x, int y) { return off[x] < off[y]; });
  }
  for (int i = 0; i + 1 < nsys; ++i) {
    const int a = sorted ? i : order[i], b = sorted ? i + 1 : order[i + 1];
    if (off[a] + len(a) > off[b]) {
      set_error("the %s of systems %d and %d overlap", kind == kSolve ? "solutions" : "inverses", a, b);
      return SIROCCO_EINVAL;
    }
  }
  return 0;
}

static int plan_build(sirocco_plan** out, int kind, int nsys, const int* n, const int64_t* offA,
                      const int64_t* offv, int mode, bool alloc_scratch = true) {
  *out = nullptr;
  if (nsys < 0 || (nsys > 0 && (!n || !offA || (kind == kSolve && !offv)))) {
    set_error("invalid plan arguments");
    return SIROCCO_EINVAL;
  }
  if (kind != kSolve && kind != kInvert) {
    set_error("kind must be 0 (solve) or 1 (invert)");
    return SIROCCO_EINVAL;
  }
  if (mode != SIROCCO_FP64 && mode != SIROCCO_MIXED && mode != SIROCCO_FAST) {
    set_error("unknown precision mode %d", mode);
    return SIROCCO_EMODE;
  }
  if (int rc = check_layout(kind, nsys, n, offA, offv)) return rc;
  std::unique_ptr<sirocco_plan, void (*)(sirocco_plan*)> p(new sirocco_plan(), plan_free);
  p->kind = kind;
  p->mode = mode;
  p->nsys = nsys;
  SS_CUDA(cudaGetDevice(&p->device));
  SS_CUDA(cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device));

  // bucket the systems: key = (family, class); global family sorted by size.
  // Certified inverses (SIROCCO_FAST) go to the Gauss-Jordan classes; each also
  // has a place in the fallback list of its exact class (small or CTA family).
  const bool cert = (kind == kInvert && mode == SIROCCO_FAST);
  std::vector<int> small_l[kSmallClasses], cta_l[kCtaClasses], glob_l, cgj_l[kCgjClasses], cgjl_l;
  int small_fb[kSmallClasses] = {}, cta_fb[kCtaClasses] = {};
  for (int s = 0; s < nsys; ++s) {
    const int ns = n[s];
    if (ns < 1 || ns > SIROCCO_MAX_N) {
      set_error("system %d has order %d (supported 1..%d)", s, ns, SIROCCO_MAX_N);
      return ns < 1 ? SIROCCO_EINVAL : SIROCCO_ESIZE;
    }
    p->totA = std::max<int64_t>(p->totA, offA[s] + int64_t(ns) * ns);
    if (kind == kSolve) p->totV = std::max<int64_t>(p->totV, offv[s] + ns);
    int c;
    if (cert && (c = cgj_class(ns)) >= 0) {
      cgj_l[c].push_back(s);
      int e;
      if ((e = small_class(ns)) >= 0) small_fb[e]++;
      else cta_fb[cta_class(ns)]++;
      continue;
    }
    if (cert && ns > kCgjP[kCgjClasses - 1]) {
      cgjl_l.push_back(s);
      cta_fb[cta_class(ns)]++;
      continue;
    }
    if ((c = small_class(ns)) >= 0) small_l[c].push_back(s);
    else if ((c = cta_class(ns)) >= 0) cta_l[c].push_back(s);
    else glob_l.push_back(s);
  }
  // fallback lists: one per exact class that certified systems belong to
  int small_fbi[kSmallClasses], cta_fbi[kCtaClasses];
  std::vector<int> xcls;
  if (cert) {
    int off = 0;
    auto add_fb = [&](int cnt) {
      if (cnt == 0) return -1;
      p->fb_off.push_back(off);
      off += cnt;
      return p->nfb++;
    };
    for (int e = 0; e < kSmallClasses; ++e) small_fbi[e] = add_fb(small_fb[e]);
    for (int e = 0; e < kCtaClasses; ++e) cta_fbi[e] = add_fb(cta_fb[e]);
    if (p->nfb > 0) {
      xcls.assign(nsys, -1);
      for (int c = 0; c < kCgjClasses; ++c)
        for (int s : cgj_l[c]) {
          const int e = small_class(n[s]);
          xcls[s] = (e >= 0) ? small_fbi[e] : cta_fbi[cta_class(n[s])];
        }
      for (int s : cgjl_l) xcls[s] = cta_fbi[cta_class(n[s])];
      p->fb_off.push_back(off);   // total size of the lists
    }
  }
  // largest systems first within the global bucket (longest jobs start first)
  std::stable_sort(glob_l.begin(), glob_l.end(), [&](int x, int y) { return n[x] > n[y]; });
  std::stable_sort(cgjl_l.begin(), cgjl_l.end(), [&](int x, int y) { return n[x] > n[y]; });

  std::vector<int> list;
  list.reserve(nsys);
  int64_t scratch_elems = 0;
  // a bucket serves either systems of the plan's list (count of them) or, in
  // phase 2, fallback list fb (at most count entries, filled on the device)
  auto add_bucket_n = [&](Family fam, int cls, const std::vector<int>* l, int fb, int cnt) -> int {
    if (cnt == 0) return 0;
    Bucket b{};
    b.fam = fam;
    b.cls = cls;
    b.count = cnt;
    b.phase = (fb >= 0) ? 2 : 1;
    b.fb = fb;
    b.list_off = int(list.size());
    if (l) list.insert(list.end(), l->begin(), l->end());
    b.q = -1;
    if (fam == kFamCgj) b.spec = cgj_spec(cls);
    else if (fam == kFamCgjL) {
      b.spec = cgjl_spec();
      b.q = p->nq++;
    }
    else if (fam == kFamSmall) b.spec = (kind == kSolve) ? small_spec<kSolve>(cls, mode) : small_spec<kInvert>(cls, mode);
    else if (fam == kFamCta) b.spec = (kind == kSolve) ? cta_spec<kSolve>(cls) : cta_spec<kInvert>(cls);
    else b.spec = (kind == kSolve) ? global_spec<kSolve>(cls) : global_spec<kInvert>(cls);
    int rc = finish_spec(b.spec);
    if (rc) return rc;
    const int blocks_needed = (b.count + b.spec.sys_per_block - 1) / b.spec.sys_per_block;
    b.grid = std::max(1, std::min(blocks_needed * b.spec.cluster, b.spec.max_ctas));
    if (fam == kFamGlobal && kind == kSolve) {
      b.slab = (int64_t(cls) * cls + 31) / 32 * 32;
      b.scratch_off = scratch_elems;
      scratch_elems += b.slab * b.grid;
    }
    if (fam == kFamCta && b.spec.work_slab > 0) {
      b.slab = b.spec.work_slab;
      b.scratch_off = scratch_elems;
      scratch_elems += b.slab * b.grid;
    }
    p->buckets.push_back(b);
    return 0;
  };
  auto add_bucket = [&](Family fam, int cls, const std::vector<int>& l) -> int {
    return add_bucket_n(fam, cls, &l, -1, int(l.size()));
  };
  int rc = 0;
  if (!glob_l.empty() && (rc = add_bucket(kFamGlobal, n[glob_l.front()], glob_l))) return rc;
  if ((rc = add_bucket(kFamCgjL, 0, cgjl_l))) return rc;
  for (int c = kCgjClasses - 1; c >= 0; --c)
    if ((rc = add_bucket(kFamCgj, c, cgj_l[c]))) return rc;
  for (int c = kCtaClasses - 1; c >= 0; --c)
    if ((rc = add_bucket(kFamCta, c, cta_l[c]))) return rc;
  for (int c = kSmallClasses - 1; c >= 0; --c)
    if ((rc = add_bucket(kFamSmall, c, small_l[c]))) return rc;
  if (cert) {
    for (int c = kCtaClasses - 1; c >= 0; --c)
      if (cta_fbi[c] >= 0 && (rc = add_bucket_n(kFamCta, c, nullptr, cta_fbi[c], cta_fb[c]))) return rc;
    for (int c = kSmallClasses - 1; c >= 0; --c)
      if (small_fbi[c] >= 0 && (rc = add_bucket_n(kFamSmall, c, nullptr, small_fbi[c], small_fb[c]))) return rc;
  }

  if (nsys > 0) {
    SS_CUDA(cudaMalloc(&p->d_n, sizeof(int) * nsys));
    SS_CUDA(cudaMalloc(&p->d_offA, sizeof(int64_t) * nsys));
    SS_CUDA(cudaMalloc(&p->d_list, sizeof(int) * nsys));
    SS_CUDA(cudaMemcpy(p->d_n, n, sizeof(int) * nsys, cudaMemcpyHostToDevice));
    SS_CUDA(cudaMemcpy(p->d_offA, offA, sizeof(int64_t) * nsys, cudaMemcpyHostToDevice));
    SS_CUDA(cudaMemcpy(p->d_list, list.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice));
    if (kind == kSolve) {
      SS_CUDA(cudaMalloc(&p->d_offv, sizeof(int64_t) * nsys));
      SS_CUDA(cudaMemcpy(p->d_offv, offv, sizeof(int64_t) * nsys, cudaMemcpyHostToDevice));
    }
    if (p->nfb + p->nq > 0) {
      SS_CUDA(cudaMalloc(&p->d_fbcount, sizeof(int) * (p->nfb + p->nq)));
      SS_CUDA(cudaMemset(p->d_fbcount, 0, sizeof(int) * (p->nfb + p->nq)));
    }
    if (p->nfb > 0) {
      SS_CUDA(cudaMalloc(&p->d_xcls, sizeof(int) * nsys));
      SS_CUDA(cudaMemcpy(p->d_xcls, xcls.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice));
      SS_CUDA(cudaMalloc(&p->d_fboff, sizeof(int) * p->fb_off.size()));
      SS_CUDA(cudaMemcpy(p->d_fboff, p->fb_off.data(), sizeof(int) * p->fb_off.size(), cudaMemcpyHostToDevice));
      SS_CUDA(cudaMalloc(&p->d_fblist, sizeof(int) * std::max(1, p->fb_off.back())));
    }
  }
  p->scratch_elems = scratch_elems;
  p->own_scratch = alloc_scratch;
  if (alloc_scratch && scratch_elems > 0) SS_CUDA(cudaMalloc(&p->d_scratch, sizeof(double) * scratch_elems));
  // one side stream per bucket of a phase beyond the first
  size_t per_phase[3] = {0, 0, 0};
  for (auto& b : p->buckets) per_phase[b.phase]++;
  for (size_t i = 1; i < std::max(per_phase[1], per_phase[2]); ++i) {
    cudaStream_t st;
    SS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    p->side.push_back(st);
    cudaEvent_t e;
    SS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    p->ev.push_back(e);
  }
  SS_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
  *out = p.release();
  return 0;
}

static int launch_bucket(const sirocco_plan* p, const Bucket& b, const double* A, const double* bvec,
                         double* out, int* status, int* diag, cudaStream_t st) {
  BatchView v;
  v.n = p->d_n;
  v.offA = p->d_offA;
  v.offv = p->d_offv;
  v.A = A;
  v.b = bvec;
  v.out = out;
  v.status = status;
  v.diag = diag;
  v.list = p->d_list + b.list_off;
  v.count = b.count;
  if (b.fb >= 0) {
    v.list = p->d_fblist + p->fb_off[b.fb];
    v.count_dev = p->d_fbcount + b.fb;
  }
  if (b.fam == kFamCgjL) {
    CertArgs ca{p->d_xcls, p->d_fboff, p->d_fblist, p->d_fbcount};
    CertEpi ep = p->epi;
    int* queue = p->d_fbcount + p->nfb + b.q;
    void* args[] = {&v, &ca, &ep, &queue};
    SS_CUDA(cudaLaunchKernel(b.spec.fn, dim3(b.grid), dim3(b.spec.threads), args, b.spec.dyn_smem, st));
  } else if (b.fam == kFamCgj) {
    CertArgs ca{p->d_xcls, p->d_fboff, p->d_fblist, p->d_fbcount};
    CertEpi ep = p->epi;
    void* args[] = {&v, &ca, &ep};
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = unsigned(b.spec.cluster);
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(unsigned(b.grid));
    cfg.blockDim = dim3(unsigned(b.spec.threads));
    cfg.dynamicSmemBytes = b.spec.dyn_smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = b.spec.cluster > 1 ? 1 : 0;
    SS_CUDA(cudaLaunchKernelExC(&cfg, b.spec.fn, args));
  } else if (b.fam == kFamGlobal) {
    int nmax = b.cls;
    double* scratch = p->d_scratch ? p->d_scratch + b.scratch_off : nullptr;
    int64_t slab = b.slab;
    void* args[] = {&v, &nmax, &scratch, &slab};
    SS_CUDA(cudaLaunchKernel(b.spec.fn, dim3(b.grid), dim3(b.spec.threads), args, b.spec.dyn_smem, st));
  } else if (b.fam == kFamCta) {
    double* work = (b.slab > 0 && p->d_scratch) ? p->d_scratch + b.scratch_off : nullptr;
    void* args[] = {&v, &work};
    SS_CUDA(cudaLaunchKernel(b.spec.fn, dim3(b.grid), dim3(b.spec.threads), args, b.spec.dyn_smem, st));
  } else if (b.fam == kFamSmall && p->mode == SIROCCO_MIXED && p->kind == kSolve) {
    MixedParams mp = default_mixed_params();
    void* args[] = {&v, &mp};
    SS_CUDA(cudaLaunchKernel(b.spec.fn, dim3(b.grid), dim3(b.spec.threads), args, b.spec.dyn_smem, st));
  } else {
    void* args[] = {&v};
    SS_CUDA(cudaLaunchKernel(b.spec.fn, dim3(b.grid), dim3(b.spec.threads), args, b.spec.dyn_smem, st));
  }
  return 0;
}

// The buckets of one phase, forked onto the side streams and joined back into st.
static int run_phase(sirocco_plan* p, int phase, const double* A, const double* bvec, double* out, int* status,
                     int* diag, cudaStream_t st) {
  std::vector<const Bucket*> bs;
  for (auto& b : p->buckets)
    if (b.phase == phase) bs.push_back(&b);
  if (bs.empty()) return 0;
  if (bs.size() == 1) return launch_bucket(p, *bs[0], A, bvec, out, status, diag, st);
  SS_CUDA(cudaEventRecord(p->ev_fork, st));
  for (size_t i = 1; i < bs.size(); ++i) SS_CUDA(cudaStreamWaitEvent(p->side[i - 1], p->ev_fork, 0));
  int rc = launch_bucket(p, *bs[0], A, bvec, out, status, diag, st);
  if (rc) return rc;
  for (size_t i = 1; i < bs.size(); ++i) {
    rc = launch_bucket(p, *bs[i], A, bvec, out, status, diag, p->side[i - 1]);
    if (rc) return rc;
    SS_CUDA(cudaEventRecord(p->ev[i - 1], p->side[i - 1]));
  }
  for (size_t i = 1; i < bs.size(); ++i) SS_CUDA(cudaStreamWaitEvent(st, p->ev[i - 1], 0));
  return 0;
}

static int plan_run(sirocco_plan* p, const double* A, const double* bvec, double* out, int* status,
                    int* diag, cudaStream_t st) {
  if (p->buckets.empty()) return 0;
  if (p->nfb + p->nq > 0) SS_CUDA(cudaMemsetAsync(p->d_fbcount, 0, sizeof(int) * size_t(p->nfb + p->nq), st));
  int rc = run_phase(p, 1, A, bvec, out, status, diag, st);
  if (rc) return rc;
  return run_phase(p, 2, A, bvec, out, status, diag, st);
}

// -------------------------------------------------------- per-thread context --
static uint64_t layout_hash(int kind, int mode, int nsys, const int* n, const int64_t* offA, const int64_t* offv) {
  uint64_t h = 1469598103934665603ull ^ (uint64_t(kind) << 8) ^ (uint64_t(mode) << 16) ^ (uint64_t(nsys) << 24);
  auto mix = [&](uint64_t x) { h ^= x + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2); };
  for (int s = 0; s < nsys; ++s) {
    mix(uint64_t(uint32_t(n[s])));
    mix(uint64_t(offA[s]));
    if (offv) mix(uint64_t(offv[s]));
  }
  return h;
}

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  int ensure(size_t want) {
    if (want <= bytes) return 0;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
      set_error("cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
      return int(e);
    }
    bytes = want;
    return 0;
  }
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
};

// A packed host batch split into chunks of consecutive systems, each with its
// own plan, so that the copies of one chunk overlap the kernels of another.
struct Pipeline {
  struct Chunk {
    int s0, s1;
    int64_t a0, a1, v0, v1;   // element ranges of A / out and of b / x
    sirocco_plan* plan;
  };
  std::vector<Chunk> chunks;
  // chunk k runs on pipeline stream k % kPipeStreams, after the chunks before it
  // on that stream: one workspace per stream serves all of that stream's chunks
  double* scratch = nullptr;
  ~Pipeline() {
    for (auto& c : chunks) plan_free(c.plan);
    cudaFree(scratch);
  }
};

#ifndef SS_CHUNK_MIB
#define SS_CHUNK_MIB 16   // smallest host pipeline chunk
#endif
#ifndef SS_PIPE_STREAMS
#define SS_PIPE_STREAMS 4 // host pipeline streams
#endif
constexpr int kPipeStreams = SS_PIPE_STREAMS;
constexpr size_t kPlanCache = 16;                      // plans cached per thread
constexpr int64_t kPlanWorkBytes = int64_t(8) << 30;   // workspace the cached plans may hold
constexpr int64_t kChunkBytes = int64_t(SS_CHUNK_MIB) << 20;

constexpr int kPipeChunks = 12;                        // chunks a large batch is cut into
constexpr int kChunkSysPerSM = 4;                      // systems per SM a chunk holds at least
constexpr int64_t kMaxChunkBytes = int64_t(4) << 30;

// Host pipeline chunk size for a batch of `total` bytes and nsys systems:
// about a twelfth of the batch, but at least the bytes of 4 systems per SM
// (of the batch's average size) so that every chunk's launch still fills the
// GPU, within [SS_CHUNK_MIB, 4 GiB].  Copies of the other chunks overlap a
// chunk's kernels.  (Config-4-like batches, 2,048 matrices of order 256-1024:
// 16 MiB chunks hold two or three matrices and ran at 660 systems/s end to end;
// chunks of a twelfth, 4,800/s; of a quarter, 8,300/s.)  SIROCCO_CHUNK_MIB
// fixes the size instead (read once).
static int64_t chunk_bytes(int64_t total, int nsys, int sms) {
  static const int64_t fixed = [] {
    const char* e = std::getenv("SIROCCO_CHUNK_MIB");
    const long m = e ? std::strtol(e, nullptr, 10) : 0;
    return (m > 0 && m <= 4096) ? int64_t(m) << 20 : int64_t(0);
  }();
  if (fixed > 0) return fixed;
  const int64_t fill = nsys > 0 ? total / nsys * kChunkSysPerSM * sms : 0;
  return std::min(kMaxChunkBytes, std::max({kChunkBytes, total / kPipeChunks, fill}));
}

struct Context {
  int device = -1;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t pipe[kPipeStreams] = {};
  cudaEvent_t pipe_ev[kPipeStreams] = {};
  std::unordered_map<uint64_t, sirocco_plan*> plans;
  std::vector<uint64_t> plan_order;
  std::unordered_map<uint64_t, std::unique_ptr<Pipeline>> pipes;
  std::vector<uint64_t> pipe_order;
  DevBuf bA, bb, bx, bst;
  DevBuf bR, bC, bOv, bN, bOa, bQs, bQl, bQz, bQt;   // macro-atom epilogue and draws
  DevBuf bIT, bI64, bID, bIL, bIS, bIA, bIB, bIX, bISt;   // ion rate-matrix assembly
  DevBuf bMT, bMD, bMN, bMR;                              // macro-atom jump-matrix assembly
  int mode = SIROCCO_FP64;
  ~Context() { release(); }
  void release() {
    for (auto& kv : plans) plan_free(kv.second);
    plans.clear();
    plan_order.clear();
    pipes.clear();
    pipe_order.clear();
    for (int i = 0; i < kPipeStreams; ++i) {
      if (pipe[i]) cudaStreamDestroy(pipe[i]);
      if (pipe_ev[i]) cudaEventDestroy(pipe_ev[i]);
      pipe[i] = nullptr;
      pipe_ev[i] = nullptr;
    }
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    device = -1;
  }
  int init() {
    int dev = 0;
    SS_CUDA(cudaGetDevice(&dev));
    if (device == dev && stream) return 0;
    release();
    SS_CUDA(cudaSetDevice(dev));
    SS_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    SS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    for (int i = 0; i < kPipeStreams; ++i) {
      SS_CUDA(cudaStreamCreateWithFlags(&pipe[i], cudaStreamNonBlocking));
      SS_CUDA(cudaEventCreateWithFlags(&pipe_ev[i], cudaEventDisableTiming));
    }
    device = dev;
    return 0;
  }
  // chunked plans of a packed layout (systems stored one after another)
  int get_pipeline(int kind, int nsys, const int* n, const int64_t* offA, const int64_t* offv, int md,
                   Pipeline** out) {
    const uint64_t h = layout_hash(kind, md, nsys, n, offA, offv) ^ 0x5bd1e995ull;
    auto it = pipes.find(h);
    if (it != pipes.end()) {
      *out = it->second.get();
      return 0;
    }
    std::unique_ptr<Pipeline> pl(new Pipeline());
    std::vector<int64_t> ra, rv;
    const int64_t cb = chunk_bytes(nsys > 0 ? 8 * (offA[nsys - 1] + int64_t(n[nsys - 1]) * n[nsys - 1] - offA[0]) : 0,
                                   nsys, num_sms);
    int s0 = 0;
    while (s0 < nsys) {
      int s1 = s0;
      int64_t bytes = 0;
      while (s1 < nsys && (s1 == s0 || bytes < cb)) {
        bytes += int64_t(n[s1]) * n[s1] * 8;
        ++s1;
      }
      Pipeline::Chunk c;
      c.s0 = s0;
      c.s1 = s1;
      c.a0 = offA[s0];
      c.a1 = offA[s1 - 1] + int64_t(n[s1 - 1]) * n[s1 - 1];
      c.v0 = offv ? offv[s0] : 0;
      c.v1 = offv ? offv[s1 - 1] + n[s1 - 1] : 0;
      ra.resize(s1 - s0);
      rv.resize(s1 - s0);
      for (int s = s0; s < s1; ++s) {
        ra[s - s0] = offA[s] - c.a0;
        rv[s - s0] = offv ? offv[s] - c.v0 : 0;
      }
      c.plan = nullptr;
      int rc = plan_build(&c.plan, kind, s1 - s0, n + s0, ra.data(), offv ? rv.data() : nullptr, md, false);
      if (rc) {
        plan_free(c.plan);
        return rc;
      }
      pl->chunks.push_back(c);
      s0 = s1;
    }
    int64_t per_stream = 0;
    for (auto& c : pl->chunks) per_stream = std::max(per_stream, c.plan->scratch_elems);
    if (per_stream > 0) {
      SS_CUDA(cudaMalloc(&pl->scratch, sizeof(double) * per_stream * kPipeStreams));
      for (size_t k = 0; k < pl->chunks.size(); ++k)
        pl->chunks[k].plan->d_scratch = pl->scratch + per_stream * int64_t(k % kPipeStreams);
    }
    if (pipe_order.size() >= 8) {
      pipes.erase(pipe_order.front());
      pipe_order.erase(pipe_order.begin());
    }
    *out = pl.get();
    pipes[h] = std::move(pl);
    pipe_order.push_back(h);
    return 0;
  }
  int get_plan(int kind, int nsys, const int* n, const int64_t* offA, const int64_t* offv, int md,
               sirocco_plan** out) {
    const uint64_t h = layout_hash(kind, md, nsys, n, offA, offv);
    auto it = plans.find(h);
    if (it != plans.end()) {
      // most recently used last
      plan_order.erase(std::find(plan_order.begin(), plan_order.end(), h));
      plan_order.push_back(h);
      *out = it->second;
      return 0;
    }
    int rc = plan_build(out, kind, nsys, n, offA, offv, md);
    if (rc) return rc;
    // at most kPlanCache plans, and no more than kPlanWorkBytes of workspace
    // held by cached plans besides the new one: least recently used go first
    auto held = [&]() {
      int64_t b = 0;
      for (auto& kv : plans) b += kv.second->scratch_elems * int64_t(sizeof(double));
      return b;
    };
    while (!plan_order.empty() && (plan_order.size() >= kPlanCache ||
                                   held() + (*out)->scratch_elems * int64_t(sizeof(double)) > kPlanWorkBytes)) {
      auto old = plans.find(plan_order.front());
      if (old != plans.end()) {
        plan_free(old->second);
        plans.erase(old);
      }
      plan_order.erase(plan_order.begin());
    }
    plans[h] = *out;
    plan_order.push_back(h);
    return 0;
  }
};

static thread_local std::unique_ptr<Context> g_ctx;

static Context* ctx() {
  if (!g_ctx) g_ctx.reset(new Context());
  return g_ctx.get();
}

// page-locked host memory: a copy into it does not block the host
static bool is_pinned_host(const void* ptr) {
  if (!ptr) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

static bool is_device_ptr(const void* ptr) {
  if (!ptr) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

static int run_batched(int kind, int nsys, const int* n, const int64_t* offA, const double* A,
                       const int64_t* offv, const double* b, double* out, int* status, int md) {
  if (nsys == 0) return 0;
  if (nsys < 0 || !n || !offA || !A || !out || !status || (kind == kSolve && (!offv || !b))) {
    set_error("invalid batched arguments");
    return SIROCCO_EINVAL;
  }
  if (int rc = check_layout(kind, nsys, n, offA, offv)) return rc;
  Context* c = ctx();
  int rc = c->init();
  if (rc) return rc;
  sirocco_plan* p = nullptr;
  rc = c->get_plan(kind, nsys, n, offA, kind == kSolve ? offv : nullptr, md, &p);
  if (rc) return rc;
  const bool dev = is_device_ptr(A);
  if (dev) {
    rc = plan_run(p, A, b, out, status, nullptr, c->stream);
    if (rc) return rc;
    SS_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
  }
  const size_t bytesA = sizeof(double) * size_t(p->totA);
  const size_t bytesV = sizeof(double) * size_t(p->totV);
  if ((rc = c->bA.ensure(bytesA)) || (rc = c->bst.ensure(sizeof(int) * size_t(nsys)))) return rc;
  if (kind == kSolve) {
    if ((rc = c->bb.ensure(bytesV)) || (rc = c->bx.ensure(bytesV))) return rc;
  } else if ((rc = c->bx.ensure(bytesA))) {
    return rc;
  }
  double* dA = static_cast<double*>(c->bA.ptr);
  double* db = static_cast<double*>(c->bb.ptr);
  double* dx = static_cast<double*>(c->bx.ptr);
  int* dst = static_cast<int*>(c->bst.ptr);
  bool packed = true;
  for (int s = 0; s + 1 < nsys && packed; ++s) {
    packed = offA[s + 1] == offA[s] + int64_t(n[s]) * n[s] && (kind != kSolve || offv[s + 1] == offv[s] + n[s]);
  }
  if (packed && bytesA > size_t(2 * chunk_bytes(int64_t(bytesA), nsys, c->num_sms))) {
    // chunked pipeline: the copies of one chunk overlap the kernels of the others
    Pipeline* pl = nullptr;
    rc = c->get_pipeline(kind, nsys, n, offA, kind == kSolve ? offv : nullptr, md, &pl);
    if (rc) return rc;
    // a device-to-host copy into pageable memory would block the host until the
    // chunk's kernel finished and stall the upload of the next chunks: such
    // results are fetched once, after the last chunk
    const bool out_pinned = is_pinned_host(out), st_pinned = is_pinned_host(status);
    SS_CUDA(cudaEventRecord(c->pipe_ev[0], c->stream));
    for (int i = 0; i < kPipeStreams; ++i) SS_CUDA(cudaStreamWaitEvent(c->pipe[i], c->pipe_ev[0], 0));
    for (size_t k = 0; k < pl->chunks.size(); ++k) {
      const Pipeline::Chunk& ch = pl->chunks[k];
      cudaStream_t st = c->pipe[k % kPipeStreams];
      const size_t na = size_t(ch.a1 - ch.a0), nv = size_t(ch.v1 - ch.v0), ns = size_t(ch.s1 - ch.s0);
      SS_CUDA(cudaMemcpyAsync(dA + ch.a0, A + ch.a0, na * sizeof(double), cudaMemcpyHostToDevice, st));
      if (kind == kSolve) SS_CUDA(cudaMemcpyAsync(db + ch.v0, b + ch.v0, nv * sizeof(double), cudaMemcpyHostToDevice, st));
      double* xo = (kind == kSolve) ? dx + ch.v0 : dx + ch.a0;
      rc = plan_run(ch.plan, dA + ch.a0, db + ch.v0, xo, dst + ch.s0, nullptr, st);
      if (rc) return rc;
      if (out_pinned) {
        if (kind == kSolve) SS_CUDA(cudaMemcpyAsync(out + ch.v0, xo, nv * sizeof(double), cudaMemcpyDeviceToHost, st));
        else SS_CUDA(cudaMemcpyAsync(out + ch.a0, xo, na * sizeof(double), cudaMemcpyDeviceToHost, st));
      }
      if (st_pinned) SS_CUDA(cudaMemcpyAsync(status + ch.s0, dst + ch.s0, ns * sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    for (int i = 0; i < kPipeStreams; ++i) SS_CUDA(cudaStreamSynchronize(c->pipe[i]));
    if (!out_pinned) SS_CUDA(cudaMemcpy(out, dx, kind == kSolve ? bytesV : bytesA, cudaMemcpyDeviceToHost));
    if (!st_pinned) SS_CUDA(cudaMemcpy(status, dst, sizeof(int) * size_t(nsys), cudaMemcpyDeviceToHost));
    return 0;
  }
  SS_CUDA(cudaMemcpyAsync(dA, A, bytesA, cudaMemcpyHostToDevice, c->stream));
  if (kind == kSolve) SS_CUDA(cudaMemcpyAsync(db, b, bytesV, cudaMemcpyHostToDevice, c->stream));
  rc = plan_run(p, dA, db, dx, dst, nullptr, c->stream);
  if (rc) return rc;
  SS_CUDA(cudaMemcpyAsync(out, dx, kind == kSolve ? bytesV : bytesA, cudaMemcpyDeviceToHost, c->stream));
  SS_CUDA(cudaMemcpyAsync(status, dst, sizeof(int) * size_t(nsys), cudaMemcpyDeviceToHost, c->stream));
  SS_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// ------------------------------------------------------------ macro atoms --
// B = N^-1 diag(R) per cell and the row running totals of B, after the
// GSL-exact FP64 inverse (the reference's calc_matom_matrix,
// source/macro_accelerate.c:311-334, and the walk of
// matom_deactivation_from_matrix, :995-1008).
static int run_matom(int nsys, const int* n, const int64_t* offA, const int64_t* offv, const double* N,
                     const double* R, double* B, double* C, int* status) {
  if (nsys == 0) return 0;
  if (nsys < 0 || !n || !offA || !offv || !N || !R || !B || !status) {
    set_error("invalid macro-atom arguments");
    return SIROCCO_EINVAL;
  }
  if (int rc = check_layout(kInvert, nsys, n, offA, nullptr)) return rc;
  for (int s = 0; s < nsys; ++s)
    if (offv[s] < 0) {
      set_error("cell %d has a negative offset of its deactivation rates", s);
      return SIROCCO_EINVAL;
    }
  Context* c = ctx();
  int rc = c->init();
  if (rc) return rc;
  // SIROCCO_FAST: certified inverses with the epilogue fused into their kernel;
  // otherwise GSL-exact inverses followed by the epilogue kernel
  const int md = (c->mode == SIROCCO_FAST) ? SIROCCO_FAST : SIROCCO_FP64;
  sirocco_plan* p = nullptr;
  rc = c->get_plan(kInvert, nsys, n, offA, nullptr, md, &p);
  if (rc) return rc;
  const bool fused = (md == SIROCCO_FAST);
  int64_t totV = 0;
  int maxn = 0;
  for (int s = 0; s < nsys; ++s) {
    totV = std::max<int64_t>(totV, offv[s] + n[s]);
    maxn = std::max(maxn, n[s]);
  }
  // blocks that fit 48 KB of shared memory are staged there (coalesced traffic)
  const size_t tile_bytes = sizeof(double) * size_t(maxn) * size_t(maxn);
  const bool tiled = tile_bytes <= size_t(48) << 10;
  // the epilogue kernel over every system, or (fused) over the systems that
  // the GSL-exact kernels served: their buckets' lists and the fallback lists
  auto epilogue_on = [&](double* Bp, const double* Rp, double* Cp, const int* stp, EpiList el, int cnt) -> int {
    const int grid = std::max(1, std::min(cnt, p->num_sms * 16));
    const int64_t* dOv = static_cast<const int64_t*>(c->bOv.ptr);
    if (tiled)
      matom_epilogue_tile_kernel<<<grid, 128, tile_bytes, c->stream>>>(nsys, p->d_n, p->d_offA, dOv, Bp, Rp, Cp, stp,
                                                                       el);
    else
      matom_epilogue_kernel<<<grid, 128, 0, c->stream>>>(nsys, p->d_n, p->d_offA, dOv, Bp, Rp, Cp, stp, el);
    SS_CUDA(cudaGetLastError());
    return 0;
  };
  auto epilogue = [&](double* Bp, const double* Rp, double* Cp, const int* stp) -> int {
    if (!fused) return epilogue_on(Bp, Rp, Cp, stp, EpiList{}, nsys);
    for (const Bucket& b : p->buckets) {
      if (b.fam == kFamCgj || b.fam == kFamCgjL) continue;
      EpiList el;
      if (b.fb >= 0) {
        el.list = p->d_fblist + p->fb_off[b.fb];
        el.count_dev = p->d_fbcount + b.fb;
      } else {
        el.list = p->d_list + b.list_off;
        el.count = b.count;
      }
      if (int r = epilogue_on(Bp, Rp, Cp, stp, el, b.count)) return r;
    }
    return 0;
  };
  // the plan run with the certified kernels writing B (and C) themselves
  auto run_plan = [&](const double* Np, double* Bp, const double* Rp, double* Cp, int* stp) -> int {
    if (fused) {
      p->epi.offv = static_cast<const int64_t*>(c->bOv.ptr);
      p->epi.R = Rp;
      p->epi.C = Cp;
    }
    const int r = plan_run(p, Np, nullptr, Bp, stp, nullptr, c->stream);
    p->epi = CertEpi{};
    return r;
  };
  if ((rc = c->bOv.ensure(sizeof(int64_t) * size_t(nsys)))) return rc;
  int64_t* dOv = static_cast<int64_t*>(c->bOv.ptr);
  SS_CUDA(cudaMemcpyAsync(dOv, offv, sizeof(int64_t) * size_t(nsys), cudaMemcpyHostToDevice, c->stream));
  if (is_device_ptr(N)) {
    rc = run_plan(N, B, R, C, status);
    if (rc) return rc;
    if ((rc = epilogue(B, R, C, status))) return rc;
    SS_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
  }
  const size_t bytesA = sizeof(double) * size_t(p->totA), bytesV = sizeof(double) * size_t(totV);
  if ((rc = c->bA.ensure(bytesA)) || (rc = c->bx.ensure(bytesA)) || (rc = c->bR.ensure(bytesV)) ||
      (rc = c->bst.ensure(sizeof(int) * size_t(nsys))) || (C && (rc = c->bC.ensure(bytesA))))
    return rc;
  double* dN = static_cast<double*>(c->bA.ptr);
  double* dB = static_cast<double*>(c->bx.ptr);
  double* dR = static_cast<double*>(c->bR.ptr);
  double* dC = C ? static_cast<double*>(c->bC.ptr) : nullptr;
  int* dst = static_cast<int*>(c->bst.ptr);
  SS_CUDA(cudaMemcpyAsync(dN, N, bytesA, cudaMemcpyHostToDevice, c->stream));
  SS_CUDA(cudaMemcpyAsync(dR, R, bytesV, cudaMemcpyHostToDevice, c->stream));
  rc = run_plan(dN, dB, dR, dC, dst);
  if (rc) return rc;
  if ((rc = epilogue(dB, dR, dC, dst))) return rc;
  SS_CUDA(cudaMemcpyAsync(B, dB, bytesA, cudaMemcpyDeviceToHost, c->stream));
  if (C) SS_CUDA(cudaMemcpyAsync(C, dC, bytesA, cudaMemcpyDeviceToHost, c->stream));
  SS_CUDA(cudaMemcpyAsync(status, dst, sizeof(int) * size_t(nsys), cudaMemcpyDeviceToHost, c->stream));
  SS_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

static int run_matom_sample(int nq, int nsys, const int* n, const int64_t* offA, const double* C, const int* sys,
                            const int* level, const double* z, int* target) {
  if (nq == 0) return 0;
  if (nq < 0 || nsys < 1 || !n || !offA || !C || !sys || !level || !z || !target) {
    set_error("invalid macro-atom draw arguments");
    return SIROCCO_EINVAL;
  }
  Context* c = ctx();
  int rc = c->init();
  if (rc) return rc;
  int64_t totA = 0;
  for (int s = 0; s < nsys; ++s) {
    if (n[s] < 1) {
      set_error("system %d has order %d", s, n[s]);
      return SIROCCO_EINVAL;
    }
    totA = std::max<int64_t>(totA, offA[s] + int64_t(n[s]) * n[s]);
  }
  if ((rc = c->bN.ensure(sizeof(int) * size_t(nsys))) || (rc = c->bOa.ensure(sizeof(int64_t) * size_t(nsys))))
    return rc;
  int* dn = static_cast<int*>(c->bN.ptr);
  int64_t* doa = static_cast<int64_t*>(c->bOa.ptr);
  SS_CUDA(cudaMemcpyAsync(dn, n, sizeof(int) * size_t(nsys), cudaMemcpyHostToDevice, c->stream));
  SS_CUDA(cudaMemcpyAsync(doa, offA, sizeof(int64_t) * size_t(nsys), cudaMemcpyHostToDevice, c->stream));
  const int grid = (nq + 255) / 256;
  if (is_device_ptr(C)) {
    matom_sample_kernel<<<grid, 256, 0, c->stream>>>(nq, nsys, dn, doa, C, sys, level, z, target);
    SS_CUDA(cudaGetLastError());
    SS_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
  }
  const size_t bytesC = sizeof(double) * size_t(totA);
  if ((rc = c->bC.ensure(bytesC)) || (rc = c->bQs.ensure(sizeof(int) * size_t(nq))) ||
      (rc = c->bQl.ensure(sizeof(int) * size_t(nq))) || (rc = c->bQz.ensure(sizeof(double) * size_t(nq))) ||
      (rc = c->bQt.ensure(sizeof(int) * size_t(nq))))
    return rc;
  double* dC = static_cast<double*>(c->bC.ptr);
  int* ds = static_cast<int*>(c->bQs.ptr);
  int* dl = static_cast<int*>(c->bQl.ptr);
  double* dz = static_cast<double*>(c->bQz.ptr);
  int* dt = static_cast<int*>(c->bQt.ptr);
  SS_CUDA(cudaMemcpyAsync(dC, C, bytesC, cudaMemcpyHostToDevice, c->stream));
  SS_CUDA(cudaMemcpyAsync(ds, sys, sizeof(int) * size_t(nq), cudaMemcpyHostToDevice, c->stream));
  SS_CUDA(cudaMemcpyAsync(dl, level, sizeof(int) * size_t(nq), cudaMemcpyHostToDevice, c->stream));
  SS_CUDA(cudaMemcpyAsync(dz, z, sizeof(double) * size_t(nq), cudaMemcpyHostToDevice, c->stream));
  matom_sample_kernel<<<grid, 256, 0, c->stream>>>(nq, nsys, dn, doa, dC, ds, dl, dz, dt);
  SS_CUDA(cudaGetLastError());
  SS_CUDA(cudaMemcpyAsync(target, dt, sizeof(int) * size_t(nq), cudaMemcpyDeviceToHost, c->stream));
  SS_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// ------------------------------------------------------- ion populations --
// Lock-step n_e iteration over many cells: the loop of matrix_ion_populations
// (source/matrix_ion.c:219-382) run for every cell at once, one batched solve
// per round over the per-element blocks of all cells that have not finished.
// The reference's rate matrix is block-diagonal by element (its first row of
// each element's block is the conservation row), so LU with partial pivoting on
// the full matrix only ever meets exact zeros outside a block: the per-element
// solves give the full matrix's solution and codes bit for bit.
constexpr double kDensityMin = 1.0e-20;   // atomic.h:9
constexpr double kFracError = 0.03;       // python.h:1212
constexpr int kMaxIterations = 200;       // python.h:1211

// Elements own consecutive ion ranges that together cover every ion once.
static int check_ion_elements(int nions, int nelem, const int* elem_first, const int* elem_n, std::vector<int>& elem_of,
                              int64_t& blkA) {
  elem_of.assign(nions, -1);
  blkA = 0;
  for (int e = 0; e < nelem; ++e) {
    if (elem_n[e] < 1 || elem_first[e] < 0 || elem_first[e] + elem_n[e] > nions) {
      set_error("element %d: ions [%d, %d) outside 0..%d", e, elem_first[e], elem_first[e] + elem_n[e], nions);
      return SIROCCO_EINVAL;
    }
    for (int k = 0; k < elem_n[e]; ++k) {
      if (elem_of[elem_first[e] + k] >= 0) {
        set_error("ion %d belongs to two elements", elem_first[e] + k);
        return SIROCCO_EINVAL;
      }
      elem_of[elem_first[e] + k] = e;
    }
    blkA += int64_t(elem_n[e]) * elem_n[e];
  }
  for (int i = 0; i < nions; ++i)
    if (elem_of[i] < 0) {
      set_error("ion %d belongs to no element", i);
      return SIROCCO_EINVAL;
    }
  return 0;
}

// One round of the lock-step for the listed cells: assemble and solve their
// element systems; x receives nions populations per cell (element order), st
// the solve codes of the cell's nelem blocks.
using IonRoundFn = std::function<int(int na, const int* cells, const double* ne, const double* nh1, const double* nh2,
                                     double* x, int* st)>;

// The n_e iteration of matrix_ion_populations (source/matrix_ion.c:219-382)
// over many cells at once: each round solves every unfinished cell.
static int ion_lockstep_core(int ncell, int nions, int nelem, const int* elem_first, const int* elem_n,
                             const int* istate, int h_elem, const double* elem_dens, const std::vector<int>& elem_of,
                             double* ne, double* den, const IonRoundFn& round, int* status, int* iters) {
  std::vector<double> xne(ne, ne + ncell), cur(den, den + size_t(ncell) * nions);
  std::vector<int> active(ncell);
  for (int c = 0; c < ncell; ++c) {
    active[c] = c;
    status[c] = -2;
    iters[c] = 0;
  }
  std::vector<double> x, nh1, nh2, nea;
  std::vector<int> st;
  for (int it = 0; it < kMaxIterations && !active.empty(); ++it) {
    const int na = int(active.size());
    nea.resize(na);
    nh1.assign(na, 0.0);
    nh2.assign(na, 0.0);
    for (int i = 0; i < na; ++i) {
      const int c = active[i];
      nea[i] = xne[c];
      if (h_elem >= 0) {
        // neutral and ionised hydrogen densities for charge exchange (matrix_ion.c:228-238)
        const double* cd = &cur[size_t(c) * nions];
        const double dh = elem_dens[size_t(c) * nelem + h_elem];
        for (int k = 0; k < elem_n[h_elem]; ++k) {
          const int nn = elem_first[h_elem] + k;
          if (istate[nn] == 1) nh1[i] = cd[nn] * dh;
          if (istate[nn] == 2) nh2[i] = cd[nn] * dh;
        }
      }
    }
    x.assign(size_t(na) * nions, 0.0);
    st.assign(size_t(na) * nelem, 0);
    int rc = round(na, active.data(), nea.data(), nh1.data(), nh2.data(), x.data(), st.data());
    if (rc) return rc;
    std::vector<int> next;
    for (int i = 0; i < na; ++i) {
      const int c = active[i];
      bool singular = false;
      for (int e = 0; e < nelem; ++e) singular |= st[size_t(i) * nelem + e] == kSolveSingular;
      iters[c] = it + 1;
      if (singular) {   // matrix_ion.c:295-299: the cell keeps its old populations
        status[c] = -1;
        continue;
      }
      double* nd = &cur[size_t(c) * nions];
      const double* xi = &x[size_t(i) * nions];
      for (int nn = 0; nn < nions; ++nn) nd[nn] = xi[nn] < kDensityMin ? kDensityMin : xi[nn];
      double xnew = 0.0;
      for (int nn = 0; nn < nions; ++nn)
        xnew += nd[nn] * (istate[nn] - 1) * elem_dens[size_t(c) * nelem + elem_of[nn]];
      if (xnew < kDensityMin) xnew = kDensityMin;
      if (std::fabs((xne[c] - xnew) / xnew) < kFracError || xnew < 1.e-6) {
        status[c] = 0;
        ne[c] = xnew;
        std::copy(nd, nd + nions, den + size_t(c) * nions);
        continue;
      }
      xne[c] = (xnew + xne[c]) / 2.;
      next.push_back(c);
    }
    active.swap(next);
  }
  // cells still active ran out of iterations (matrix_ion.c:366-382): status -2, inputs kept
  return 0;
}

// The batched layout of na cells' element systems: cell i's blocks one after
// another (element order), its right-hand side and solution at i * nions.
static void ion_block_layout(int na, int nions, int nelem, const int* elem_first, const int* elem_n, int64_t blkA,
                             std::vector<int>& n, std::vector<int64_t>& offA, std::vector<int64_t>& offv) {
  const int nsys = na * nelem;
  n.resize(nsys);
  offA.resize(nsys);
  offv.resize(nsys);
  for (int i = 0, s = 0; i < na; ++i) {
    int64_t oa = int64_t(i) * blkA;
    for (int e = 0; e < nelem; ++e, ++s) {
      n[s] = elem_n[e];
      offA[s] = oa;
      offv[s] = int64_t(i) * nions + elem_first[e];
      oa += int64_t(elem_n[e]) * elem_n[e];
    }
  }
}

static int run_ion_lockstep(int ncell, int nions, int nelem, const int* elem_first, const int* elem_n,
                            const int* istate, int h_elem, const double* elem_dens, double* ne, double* den,
                            sirocco_ion_assemble_fn assemble, void* user, int* status, int* iters) {
  if (ncell == 0) return 0;
  if (ncell < 0 || nions < 1 || nelem < 1 || !elem_first || !elem_n || !istate || !elem_dens || !ne || !den ||
      !assemble || !status || !iters || h_elem >= nelem) {
    set_error("invalid lock-step arguments");
    return SIROCCO_EINVAL;
  }
  std::vector<int> elem_of;
  int64_t blkA = 0;
  int rc = check_ion_elements(nions, nelem, elem_first, elem_n, elem_of, blkA);
  if (rc) return rc;
  std::vector<double> A, b;
  std::vector<int> n;
  std::vector<int64_t> offA, offv;
  auto round = [&](int na, const int* cells, const double* nea, const double* nh1, const double* nh2, double* x,
                   int* st) -> int {
    A.assign(size_t(na) * blkA, 0.0);
    b.assign(size_t(na) * nions, 0.0);
    const int arc = assemble(user, na, cells, nea, nh1, nh2, A.data(), b.data());
    if (arc != 0) {
      set_error("assembly callback returned %d", arc);
      return SIROCCO_EINVAL;
    }
    ion_block_layout(na, nions, nelem, elem_first, elem_n, blkA, n, offA, offv);
    return run_batched(kSolve, na * nelem, n.data(), offA.data(), A.data(), offv.data(), b.data(), x, st,
                       ctx()->mode);
  };
  return ion_lockstep_core(ncell, nions, nelem, elem_first, elem_n, istate, h_elem, elem_dens, elem_of, ne, den,
                           round, status, iters);
}

// ------------------------------------------------- ion rate-matrix assembly --
// Checks a table and its rates, builds the per-ion flags and the per-ion
// lists of charge-exchange and inner-shell entries, and uploads everything for
// ion_assemble_kernel.  v gets the device pointers of everything but the
// per-round arrays.
static int ion_asm_prepare(const sirocco_ion_table* t, int ncell, const sirocco_ion_rates* r, Context* c,
                           IonAsmView& v, std::vector<int>& elem_of, int64_t& blkA) {
  if (!t || !r || t->nions < 1 || t->nelem < 1 || !t->elem_z || !t->elem_first || !t->elem_n || !t->elem_istate_max ||
      !t->ion_istate || !t->ion_di || !t->ion_dr || t->n_inner < 0 || t->n_yield < 0 || t->ncx < 0 ||
      (t->n_inner > 0 && (!t->inner_nion || !t->inner_yield)) || (t->n_yield > 0 && !t->yield_prob) ||
      (t->ncx > 0 && (!t->cx_nion1 || !t->cx_nion2)) || !r->pi || !r->rr || !r->di || !r->qr || !r->dr || !r->cxr ||
      (t->ncx > 0 && !r->cxi) || (t->n_inner > 0 && !r->inner)) {
    set_error("invalid ion table or rates");
    return SIROCCO_EINVAL;
  }
  const int nions = t->nions, nelem = t->nelem;
  int rc = check_ion_elements(nions, nelem, t->elem_first, t->elem_n, elem_of, blkA);
  if (rc) return rc;
  auto last_of = [&](int i) { const int e = elem_of[i]; return t->elem_first[e] + t->elem_n[e] - 1; };
  std::vector<int> flags(nions), zion(nions);
  for (int i = 0; i < nions; ++i) {
    const int e = elem_of[i];
    zion[i] = t->elem_z[e];
    flags[i] = (t->ion_istate[i] == t->elem_istate_max[e] ? 1 : 0) | (t->ion_di[i] > 0 ? 2 : 0) |
               (t->ion_dr[i] > 0 ? 4 : 0);
  }
  // charge-exchange ionisation against hydrogen, per ionised ion, in entry order
  std::vector<int> cx_start(nions + 1, 0), in_start(nions + 1, 0), cx_idx, in_idx, in_yield;
  std::vector<std::vector<int>> cx_of(nions), in_of(nions);
  for (int m = 0; m < t->ncx; ++m) {
    const int o = t->cx_nion1[m], p = t->cx_nion2[m];
    if (o < 0 || o >= nions || p < 0 || p >= nions) {
      set_error("charge-exchange entry %d: ions %d, %d outside 0..%d", m, o, p, nions);
      return SIROCCO_EINVAL;
    }
    if (zion[p] != 1) continue;
    if (o + 1 > last_of(o)) {
      set_error("charge-exchange entry %d ionises ion %d, the last of its element", m, o);
      return SIROCCO_EINVAL;
    }
    cx_of[o].push_back(m);
  }
  for (int m = 0; m < t->n_inner; ++m) {
    const int o = t->inner_nion[m], y = t->inner_yield[m];
    if (o < 0 || o >= nions || y < -1 || y >= t->n_yield) {
      set_error("inner-shell rate %d: ion %d or yield row %d out of range", m, o, y);
      return SIROCCO_EINVAL;
    }
    if (y == -1) continue;
    const int nel = std::min(zion[o] - t->ion_istate[o] + 1, 11);
    if (nel > 1 && o + nel - 1 > last_of(o)) {
      set_error("inner-shell rate %d of ion %d yields past its element's last ion", m, o);
      return SIROCCO_EINVAL;
    }
    in_of[o].push_back(m);
  }
  for (int i = 0; i < nions; ++i) {
    cx_start[i + 1] = cx_start[i] + int(cx_of[i].size());
    cx_idx.insert(cx_idx.end(), cx_of[i].begin(), cx_of[i].end());
    in_start[i + 1] = in_start[i] + int(in_of[i].size());
    for (int m : in_of[i]) {
      in_idx.push_back(m);
      in_yield.push_back(t->inner_yield[m]);
    }
  }
  // charge-exchange recombination writes above each ion (matrix_ion.c:579-585);
  // above a neutral ion that entry belongs to another element and must be zero
  if (t->ncx > 0)
    for (int e = 0; e < nelem; ++e) {
      if (t->elem_z[e] == 1) continue;
      const int f = t->elem_first[e];
      for (int cc = 0; cc < ncell; ++cc)
        if (r->cxr[size_t(cc) * nions + f] != 0.0) {
          set_error("cell %d: charge-exchange recombination of neutral ion %d reaches outside its element", cc, f);
          return SIROCCO_EINVAL;
        }
    }
  // the table is valid: from here on the device is needed
  if ((rc = c->init())) return rc;
  // ints: elem_first, elem_n, ion_z, ion_istate, flags, cx_start, cx_idx, in_start, in_idx, in_yield
  std::vector<int> ints;
  std::vector<size_t> io;
  auto put_i = [&](const int* p, size_t k) { io.push_back(ints.size()); ints.insert(ints.end(), p, p + k); };
  put_i(t->elem_first, nelem);
  put_i(t->elem_n, nelem);
  put_i(zion.data(), nions);
  put_i(t->ion_istate, nions);
  put_i(flags.data(), nions);
  put_i(cx_start.data(), nions + 1);
  put_i(cx_idx.data(), cx_idx.size());
  put_i(in_start.data(), nions + 1);
  put_i(in_idx.data(), in_idx.size());
  put_i(in_yield.data(), in_yield.size());
  std::vector<int64_t> boff(nelem);
  for (int e = 0, o = 0; e < nelem; ++e) {
    boff[e] = o;
    o += t->elem_n[e] * t->elem_n[e];
  }
  const size_t cn = size_t(ncell) * nions;
  std::vector<size_t> dsz = {size_t(t->n_yield) * 10, cn, cn, cn, cn, cn, cn, size_t(ncell) * t->ncx,
                             size_t(ncell) * t->n_inner};
  const double* dsrc[] = {t->yield_prob, r->pi, r->rr, r->di, r->qr, r->dr, r->cxr, r->cxi, r->inner};
  size_t dtot = 0;
  for (size_t k : dsz) dtot += k;
  if ((rc = c->bIT.ensure(sizeof(int) * std::max<size_t>(ints.size(), 1))) ||
      (rc = c->bI64.ensure(sizeof(int64_t) * nelem)) || (rc = c->bID.ensure(sizeof(double) * std::max<size_t>(dtot, 1))))
    return rc;
  int* di_ = static_cast<int*>(c->bIT.ptr);
  double* dd = static_cast<double*>(c->bID.ptr);
  SS_CUDA(cudaMemcpy(di_, ints.data(), sizeof(int) * ints.size(), cudaMemcpyHostToDevice));
  SS_CUDA(cudaMemcpy(c->bI64.ptr, boff.data(), sizeof(int64_t) * nelem, cudaMemcpyHostToDevice));
  const double* dptr[9];
  size_t off = 0;
  for (int k = 0; k < 9; ++k) {
    dptr[k] = dd + off;
    if (dsz[k] > 0) SS_CUDA(cudaMemcpy(dd + off, dsrc[k], sizeof(double) * dsz[k], cudaMemcpyHostToDevice));
    off += dsz[k];
  }
  v = IonAsmView{};
  v.nions = nions;
  v.nelem = nelem;
  v.ncx = t->ncx;
  v.n_inner = t->n_inner;
  v.elem_first = di_ + io[0];
  v.elem_n = di_ + io[1];
  v.ion_z = di_ + io[2];
  v.ion_istate = di_ + io[3];
  v.ion_flags = di_ + io[4];
  v.cx_start = di_ + io[5];
  v.cx_idx = di_ + io[6];
  v.in_start = di_ + io[7];
  v.in_idx = di_ + io[8];
  v.in_yield = di_ + io[9];
  v.blk_off = static_cast<const int64_t*>(c->bI64.ptr);
  v.blk_cell = blkA;
  v.yield = dptr[0];
  v.pi = dptr[1];
  v.rr = dptr[2];
  v.di = dptr[3];
  v.qr = dptr[4];
  v.dr = dptr[5];
  v.cxr = dptr[6];
  v.cxi = dptr[7];
  v.inner = dptr[8];
  return 0;
}

// Assembles the listed cells' element systems into the context's device
// buffers bIA (A) and bIB (b) on the context stream.
static int ion_asm_round(Context* c, IonAsmView& v, int na, const int* cells, const double* ne, const double* nh1,
                         const double* nh2) {
  int rc;
  if ((rc = c->bIL.ensure(sizeof(int) * size_t(na))) || (rc = c->bIS.ensure(sizeof(double) * 3 * size_t(na))) ||
      (rc = c->bIA.ensure(sizeof(double) * size_t(na) * size_t(v.blk_cell))) ||
      (rc = c->bIB.ensure(sizeof(double) * size_t(na) * size_t(v.nions))))
    return rc;
  double* ds = static_cast<double*>(c->bIS.ptr);
  SS_CUDA(cudaMemcpyAsync(c->bIL.ptr, cells, sizeof(int) * size_t(na), cudaMemcpyHostToDevice, c->stream));
  SS_CUDA(cudaMemcpyAsync(ds, ne, sizeof(double) * size_t(na), cudaMemcpyHostToDevice, c->stream));
  SS_CUDA(cudaMemcpyAsync(ds + na, nh1, sizeof(double) * size_t(na), cudaMemcpyHostToDevice, c->stream));
  SS_CUDA(cudaMemcpyAsync(ds + 2 * size_t(na), nh2, sizeof(double) * size_t(na), cudaMemcpyHostToDevice, c->stream));
  v.count = na;
  v.cells = static_cast<const int*>(c->bIL.ptr);
  v.ne = ds;
  v.nh1 = ds + na;
  v.nh2 = ds + 2 * size_t(na);
  v.A = static_cast<double*>(c->bIA.ptr);
  v.b = static_cast<double*>(c->bIB.ptr);
  const int64_t warps = int64_t(na) * v.nelem;
  const int64_t grid = (warps * 32 + kIonAsmThreads - 1) / kIonAsmThreads;
  ion_assemble_kernel<<<unsigned(grid), kIonAsmThreads, 0, c->stream>>>(v);
  SS_CUDA(cudaGetLastError());
  return 0;
}

static int run_ion_rate_matrices(const sirocco_ion_table* t, int ncell, const sirocco_ion_rates* r, const double* ne,
                                 const double* nh1, const double* nh2, double* A, double* b) {
  if (ncell == 0) return 0;
  if (ncell < 0 || !ne || !nh1 || !nh2 || !A || !b) {
    set_error("invalid rate-matrix arguments");
    return SIROCCO_EINVAL;
  }
  Context* c = ctx();
  int rc;
  IonAsmView v;
  std::vector<int> elem_of;
  int64_t blkA = 0;
  if ((rc = ion_asm_prepare(t, ncell, r, c, v, elem_of, blkA))) return rc;
  std::vector<int> cells(ncell);
  for (int i = 0; i < ncell; ++i) cells[i] = i;
  if ((rc = ion_asm_round(c, v, ncell, cells.data(), ne, nh1, nh2))) return rc;
  SS_CUDA(cudaMemcpyAsync(A, v.A, sizeof(double) * size_t(ncell) * size_t(blkA), cudaMemcpyDeviceToHost, c->stream));
  SS_CUDA(cudaMemcpyAsync(b, v.b, sizeof(double) * size_t(ncell) * size_t(t->nions), cudaMemcpyDeviceToHost,
                          c->stream));
  SS_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

static int run_ion_lockstep_rates(const sirocco_ion_table* t, int ncell, const sirocco_ion_rates* r, int h_elem,
                                  const double* elem_dens, double* ne, double* den, int* status, int* iters) {
  if (ncell == 0) return 0;
  if (ncell < 0 || !t || !elem_dens || !ne || !den || !status || !iters || h_elem >= t->nelem) {
    set_error("invalid lock-step arguments");
    return SIROCCO_EINVAL;
  }
  Context* c = ctx();
  int rc;
  IonAsmView v;
  std::vector<int> elem_of;
  int64_t blkA = 0;
  if ((rc = ion_asm_prepare(t, ncell, r, c, v, elem_of, blkA))) return rc;
  const int nions = t->nions, nelem = t->nelem;
  std::vector<int> n, pc;
  std::vector<int64_t> offA, offv;
  std::vector<double> pne, ph1, ph2;
  auto round = [&](int na, const int* cells, const double* nea, const double* nh1, const double* nh2, double* x,
                   int* st) -> int {
    // The active set shrinks round by round; padded to a power of two with
    // repeats of its first cell (their results are dropped) it takes at most
    // log2(ncell) + 1 layouts, whose plans stay cached.  Every system is solved
    // on its own, so the padding changes no result.
    int np2 = 1;
    while (np2 < na) np2 <<= 1;
    pc.assign(cells, cells + na);
    pne.assign(nea, nea + na);
    ph1.assign(nh1, nh1 + na);
    ph2.assign(nh2, nh2 + na);
    pc.resize(np2, cells[0]);
    pne.resize(np2, nea[0]);
    ph1.resize(np2, nh1[0]);
    ph2.resize(np2, nh2[0]);
    int rc2 = ion_asm_round(c, v, np2, pc.data(), pne.data(), ph1.data(), ph2.data());
    if (rc2) return rc2;
    if ((rc2 = c->bIX.ensure(sizeof(double) * size_t(np2) * nions)) ||
        (rc2 = c->bISt.ensure(sizeof(int) * size_t(np2) * nelem)))
      return rc2;
    ion_block_layout(np2, nions, nelem, t->elem_first, t->elem_n, blkA, n, offA, offv);
    rc2 = run_batched(kSolve, np2 * nelem, n.data(), offA.data(), v.A, offv.data(), v.b,
                      static_cast<double*>(c->bIX.ptr), static_cast<int*>(c->bISt.ptr), c->mode);
    if (rc2) return rc2;
    SS_CUDA(cudaMemcpy(x, c->bIX.ptr, sizeof(double) * size_t(na) * nions, cudaMemcpyDeviceToHost));
    SS_CUDA(cudaMemcpy(st, c->bISt.ptr, sizeof(int) * size_t(na) * nelem, cudaMemcpyDeviceToHost));
    return 0;
  };
  return ion_lockstep_core(ncell, nions, nelem, t->elem_first, t->elem_n, t->ion_istate, h_elem, elem_dens, elem_of,
                           ne, den, round, status, iters);
}

// ------------------------------------------- macro-atom jump-matrix assembly --
static int run_matom_rate_matrices(const sirocco_matom_table* t, int ncell, const sirocco_matom_rates* r, double* N,
                                   double* R) {
  if (ncell == 0) return 0;
  if (ncell < 0 || !t || !r || !N || !R || t->nlev < 1 || !t->ex || !t->bbd_start || !t->aug_start ||
      !t->bfd_start || !t->bbu_start || !t->bfu_start || t->n_kbb < 0 || t->n_kbf < 0 ||
      (t->n_kbb > 0 && !t->kbb_target) || (t->n_kbf > 0 && !t->kbf_target) || !r->kr || !r->ne) {
    set_error("invalid macro-atom table or rates");
    return SIROCCO_EINVAL;
  }
  const int nlev = t->nlev;
  // each jump list: its starts ascend from 0 and its targets are levels
  const int* starts[5] = {t->bbd_start, t->aug_start, t->bfd_start, t->bbu_start, t->bfu_start};
  const int* targets[5] = {t->bbd_target, t->aug_target, t->bfd_target, t->bbu_target, t->bfu_target};
  int cnt[5];
  for (int l = 0; l < 5; ++l) {
    if (starts[l][0] != 0) {
      set_error("jump list %d does not start at 0", l);
      return SIROCCO_EINVAL;
    }
    for (int u = 0; u < nlev; ++u)
      if (starts[l][u + 1] < starts[l][u]) {
        set_error("jump list %d: starts descend at level %d", l, u);
        return SIROCCO_EINVAL;
      }
    cnt[l] = starts[l][nlev];
    if (cnt[l] > 0 && !targets[l]) {
      set_error("jump list %d has no targets", l);
      return SIROCCO_EINVAL;
    }
    for (int j = 0; j < cnt[l]; ++j)
      if (targets[l][j] < 0 || targets[l][j] >= nlev) {
        set_error("jump list %d: target %d of jump %d outside 0..%d", l, targets[l][j], j, nlev - 1);
        return SIROCCO_EINVAL;
      }
  }
  for (int j = 0; j < t->n_kbb; ++j)
    if (t->kbb_target[j] < 0 || t->kbb_target[j] >= nlev) {
      set_error("k-packet line %d: target %d outside 0..%d", j, t->kbb_target[j], nlev - 1);
      return SIROCCO_EINVAL;
    }
  for (int j = 0; j < t->n_kbf; ++j)
    if (t->kbf_target[j] < 0 || t->kbf_target[j] >= nlev) {
      set_error("k-packet continuum %d: target %d outside 0..%d", j, t->kbf_target[j], nlev - 1);
      return SIROCCO_EINVAL;
    }
  const int n_bbd = cnt[0], n_aug = cnt[1], n_bfd = cnt[2], n_bbu = cnt[3], n_bfu = cnt[4];
  if ((n_aug > 0 && !t->aug_rate) || (n_bbd > 0 && (!r->bbd_rad || !r->bbd_coll)) ||
      (n_bfd > 0 && (!r->bfd_sp || !r->bfd_qrec)) || (n_bbu > 0 && (!r->bbu_rad || !r->bbu_coll)) ||
      (n_bfu > 0 && (!r->bfu_gamma || !r->bfu_alpha || !r->bfu_ratio || !r->bfu_qion)) ||
      (t->n_kbb > 0 && !r->kbb) || (t->n_kbf > 0 && !r->kbf)) {
    set_error("missing macro-atom coefficients");
    return SIROCCO_EINVAL;
  }
  Context* c = ctx();
  int rc = c->init();
  if (rc) return rc;
  // ints: five (starts, targets) pairs, then the k-packet targets
  std::vector<int> ints;
  std::vector<size_t> io;
  auto put_i = [&](const int* p, size_t k) {
    io.push_back(ints.size());
    if (k) ints.insert(ints.end(), p, p + k);
  };
  for (int l = 0; l < 5; ++l) {
    put_i(starts[l], size_t(nlev) + 1);
    put_i(targets[l], size_t(cnt[l]));
  }
  put_i(t->kbb_target, size_t(t->n_kbb));
  put_i(t->kbf_target, size_t(t->n_kbf));
  // doubles: ex, aug_rate, then the per-cell coefficients
  const size_t nc = size_t(ncell);
  const size_t dsz[] = {size_t(nlev), size_t(n_aug), nc * n_bbd, nc * n_bbd, nc * n_bfd, nc * n_bfd, nc * n_bbu,
                        nc * n_bbu, nc * n_bfu, nc * n_bfu, nc * n_bfu, nc * n_bfu, nc * t->n_kbb, nc * t->n_kbf,
                        nc, nc};
  const double* dsrc[] = {t->ex, t->aug_rate, r->bbd_rad, r->bbd_coll, r->bfd_sp, r->bfd_qrec, r->bbu_rad,
                          r->bbu_coll, r->bfu_gamma, r->bfu_alpha, r->bfu_ratio, r->bfu_qion, r->kbb, r->kbf, r->kr,
                          r->ne};
  constexpr int ND = int(sizeof(dsz) / sizeof(dsz[0]));
  size_t dtot = 0;
  for (size_t k : dsz) dtot += k;
  const int nr = nlev + 1;
  const bool devN = is_device_ptr(N), devR = is_device_ptr(R);
  if ((rc = c->bMT.ensure(sizeof(int) * std::max<size_t>(ints.size(), 1))) ||
      (rc = c->bMD.ensure(sizeof(double) * std::max<size_t>(dtot, 1))) ||
      (!devN && (rc = c->bMN.ensure(sizeof(double) * nc * nr * nr))) ||
      (!devR && (rc = c->bMR.ensure(sizeof(double) * nc * nr))))
    return rc;
  int* di_ = static_cast<int*>(c->bMT.ptr);
  double* dd = static_cast<double*>(c->bMD.ptr);
  SS_CUDA(cudaMemcpy(di_, ints.data(), sizeof(int) * ints.size(), cudaMemcpyHostToDevice));
  const double* dp[ND];
  size_t off = 0;
  for (int k = 0; k < ND; ++k) {
    dp[k] = dd + off;
    if (dsz[k] > 0) SS_CUDA(cudaMemcpy(dd + off, dsrc[k], sizeof(double) * dsz[k], cudaMemcpyHostToDevice));
    off += dsz[k];
  }
  MatomAsmView v{};
  v.nlev = nlev;
  v.n_bbd = n_bbd;
  v.n_aug = n_aug;
  v.n_bfd = n_bfd;
  v.n_bbu = n_bbu;
  v.n_bfu = n_bfu;
  v.n_kbb = t->n_kbb;
  v.n_kbf = t->n_kbf;
  v.bbd_start = di_ + io[0];
  v.bbd_t = di_ + io[1];
  v.aug_start = di_ + io[2];
  v.aug_t = di_ + io[3];
  v.bfd_start = di_ + io[4];
  v.bfd_t = di_ + io[5];
  v.bbu_start = di_ + io[6];
  v.bbu_t = di_ + io[7];
  v.bfu_start = di_ + io[8];
  v.bfu_t = di_ + io[9];
  v.kbb_t = di_ + io[10];
  v.kbf_t = di_ + io[11];
  v.ex = dp[0];
  v.aug_rate = dp[1];
  v.bbd_rad = dp[2];
  v.bbd_coll = dp[3];
  v.bfd_sp = dp[4];
  v.bfd_qrec = dp[5];
  v.bbu_rad = dp[6];
  v.bbu_coll = dp[7];
  v.bfu_gamma = dp[8];
  v.bfu_alpha = dp[9];
  v.bfu_ratio = dp[10];
  v.bfu_qion = dp[11];
  v.kbb = dp[12];
  v.kbf = dp[13];
  v.kr = dp[14];
  v.ne = dp[15];
  v.ncell = ncell;
  v.N = devN ? N : static_cast<double*>(c->bMN.ptr);
  v.R = devR ? R : static_cast<double*>(c->bMR.ptr);
  // a block's rows are built in shared memory when at least a warp of them fits 48 KB
  const size_t row_bytes = sizeof(double) * size_t(nr), smem_cap = size_t(48) << 10;
  int bt = kMatomAsmThreads;
  while (bt > 32 && size_t(bt) * row_bytes > smem_cap) bt -= 32;
  const bool staged = size_t(bt) * row_bytes <= smem_cap;
  if (!staged) bt = kMatomAsmThreads;
  const int64_t rows = int64_t(ncell) * nr;
  matom_assemble_kernel<<<unsigned((rows + bt - 1) / bt), bt, staged ? size_t(bt) * row_bytes : 0, c->stream>>>(
      v, staged);
  SS_CUDA(cudaGetLastError());
  if (!devN) SS_CUDA(cudaMemcpyAsync(N, v.N, sizeof(double) * nc * nr * nr, cudaMemcpyDeviceToHost, c->stream));
  if (!devR) SS_CUDA(cudaMemcpyAsync(R, v.R, sizeof(double) * nc * nr, cudaMemcpyDeviceToHost, c->stream));
  SS_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// --------------------------------------------------------- macro-atom pops --
// macro_pops (source/macro_gov.c:336-505) for one macro element over many cells:
// each round solves the level systems of every unfinished cell in one batched
// call, then applies the reference's post-processing per cell.
static int run_macro_pops(int ncell, int n, int nion, const int* ion_first, const int* ion_nlte, const double* g,
                          const unsigned char* radiative, const double* scale, sirocco_macro_assemble_fn assemble,
                          void* user, double* pop, int* status, int* iters) {
  if (ncell == 0) return 0;
  if (ncell < 0 || n < 1 || n > SIROCCO_MAX_N || nion < 1 || !ion_first || !ion_nlte || !g || !radiative ||
      !scale || !assemble || !pop || !status || !iters) {
    set_error("invalid macro_pops arguments");
    return SIROCCO_EINVAL;
  }
  for (int q = 0; q < nion; ++q)
    if (ion_first[q] < 0 || ion_nlte[q] < 0 || ion_first[q] + ion_nlte[q] > n) {
      set_error("ion %d: levels [%d, %d) outside 0..%d", q, ion_first[q], ion_first[q] + ion_nlte[q], n);
      return SIROCCO_EINVAL;
    }
  std::vector<int> active(ncell), attempt(ncell, 1);
  for (int c = 0; c < ncell; ++c) {
    active[c] = c;
    status[c] = -2;
    iters[c] = 0;
  }
  const int64_t nn = int64_t(n) * n;
  std::vector<double> A, b, x;
  std::vector<int> nv, st, att;
  std::vector<int64_t> offA, offv;
  for (int it = 1; it <= kMaxIterations && !active.empty(); ++it) {
    const int na = int(active.size());
    att.resize(na);
    for (int i = 0; i < na; ++i) att[i] = attempt[active[i]];
    A.assign(size_t(na) * nn, 0.0);
    const int arc = assemble(user, na, active.data(), att.data(), A.data());
    if (arc != 0) {
      set_error("assembly callback returned %d", arc);
      return SIROCCO_EINVAL;
    }
    // normalisation constraint in the first row, b = e_0 (macro_gov.c:401-404, 431)
    b.assign(size_t(na) * n, 0.0);
    nv.assign(na, n);
    offA.resize(na);
    offv.resize(na);
    for (int i = 0; i < na; ++i) {
      for (int k = 0; k < n; ++k) A[size_t(i) * nn + k] = 1.0;
      b[size_t(i) * n] = 1.0;
      offA[i] = int64_t(i) * nn;
      offv[i] = int64_t(i) * n;
    }
    x.assign(size_t(na) * n, 0.0);
    st.assign(na, 0);
    int rc = run_batched(kSolve, na, nv.data(), offA.data(), A.data(), offv.data(), b.data(), x.data(), st.data(),
                         ctx()->mode);
    if (rc) return rc;
    std::vector<int> next;
    for (int i = 0; i < na; ++i) {
      const int c = active[i];
      double* p = &x[size_t(i) * n];
      iters[c] = it;
      // a singular system leaves the reference's zero-filled populations
      if (st[i] == kSolveSingular) std::fill(p, p + n, 0.0);
      for (int k = 0; k < n; ++k)
        if (p[k] < kDensityMin) p[k] = 0.0;
      // population inversions between radiatively linked levels (macro_gov.c:771-804)
      for (int q = 0; q < nion; ++q) {
        const int f = ion_first[q], e = ion_first[q] + ion_nlte[q];
        for (int lo = f; lo < e; ++lo)
          for (int up = lo + 1; up < e; ++up)
            if (radiative[size_t(lo) * n + up]) {
              const double test = p[lo] * g[up] / g[lo] * 0.999999;
              if (p[up] > test) p[up] = test;
            }
      }
      // negative or non-finite ion densities or level populations (macro_gov.c:823-865)
      bool bad = false;
      for (int q = 0; q < nion; ++q) {
        const int f = ion_first[q], e = ion_first[q] + ion_nlte[q];
        double dens = 0.0;
        for (int k = f; k < e; ++k) dens += p[k];
        const double d = dens * scale[c];
        if (!std::isfinite(d) || d < 0.0) bad = true;
        for (int k = f; k < e; ++k)
          if (p[k] < 0.0 || !std::isfinite(p[k])) bad = true;
      }
      if (!bad) {
        status[c] = 0;
        std::copy(p, p + n, pop + size_t(c) * n);
      } else if (it < kMaxIterations) {
        attempt[c] = it + 1;   // the caller re-assembles with dilute estimators
        next.push_back(c);
      }
    }
    active.swap(next);
  }
  return 0;
}

// single system through the host path, honouring the reference's "output
// untouched on a singular matrix" behaviour
static int run_single(int kind, double* A, const double* b, int size, double* out, int* code) {
  if (size < 1 || !A || !out || (kind == kSolve && !b)) {
    set_error("invalid arguments");
    return SIROCCO_EINVAL;
  }
  Context* c = ctx();
  int rc = c->init();
  if (rc) return rc;
  const int nn[1] = {size};
  const int64_t oa[1] = {0}, ov[1] = {0};
  sirocco_plan* p = nullptr;
  rc = c->get_plan(kind, 1, nn, oa, kind == kSolve ? ov : nullptr, SIROCCO_FP64, &p);
  if (rc) return rc;
  const size_t bytesA = sizeof(double) * size_t(size) * size;
  const size_t bytesV = sizeof(double) * size_t(size);
  if ((rc = c->bA.ensure(bytesA)) || (rc = c->bst.ensure(sizeof(int)))) return rc;
  if ((rc = c->bb.ensure(bytesV)) || (rc = c->bx.ensure(kind == kSolve ? bytesV : bytesA))) return rc;
  double* dA = static_cast<double*>(c->bA.ptr);
  double* db = static_cast<double*>(c->bb.ptr);
  double* dx = static_cast<double*>(c->bx.ptr);
  int* dst = static_cast<int*>(c->bst.ptr);
  SS_CUDA(cudaMemcpyAsync(dA, A, bytesA, cudaMemcpyHostToDevice, c->stream));
  if (kind == kSolve) SS_CUDA(cudaMemcpyAsync(db, b, bytesV, cudaMemcpyHostToDevice, c->stream));
  rc = plan_run(p, dA, db, dx, dst, nullptr, c->stream);
  if (rc) return rc;
  SS_CUDA(cudaMemcpyAsync(code, dst, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SS_CUDA(cudaStreamSynchronize(c->stream));
  const bool write = (kind == kSolve) ? (*code != kSolveSingular) : (*code == kOk);
  if (write) SS_CUDA(cudaMemcpy(out, dx, kind == kSolve ? bytesV : bytesA, cudaMemcpyDeviceToHost));
  return 0;
}

}  // namespace ss

namespace ss {

// ---------------------------------------------------------- no-allocation --
// Scratch of solve_matrix_batched_noalloc: one n x n slab per resident CTA of the
// global-memory solve kernel, in a file-scope device array instead of cudaMalloc'd
// memory.  Every GPU that loads this library holds the array until the process
// exits; every call shares it and overwrites what the previous call left there.
constexpr int kNoAllocMaxN = SIROCCO_NOALLOC_MAX_N;
constexpr int kNoAllocSlabs = SIROCCO_NOALLOC_SLABS;
constexpr int64_t kNoAllocSlab = int64_t(kNoAllocMaxN) * kNoAllocMaxN;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlabs * kNoAllocSlab];

constexpr int kMaxDevices = 64;
static std::mutex g_noalloc_mu;
static bool g_noalloc_ready[kMaxDevices] = {};

// The array's device address on the current device.  In host code the symbol
// g_noalloc_scratch is only a host-side handle, so the address is looked up with
// that device current, on every call (the lookup is cheap, and a cached address
// would go stale if the caller reset the device).  The first call on a device
// also raises the kernel's shared-memory limit to what the largest allowed
// order needs, once, so that concurrent calls with different orders never see
// a limit below their launch.
static int noalloc_scratch(double** out, const void* fn) {
  int dev = 0;
  SS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device %d beyond the %d devices the no-allocation path tracks", dev, kMaxDevices);
    return SIROCCO_EINVAL;
  }
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ready[dev]) {
      SS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(global_smem_bytes(kNoAllocMaxN))));
      g_noalloc_ready[dev] = true;
    }
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    set_error("cudaGetSymbolAddress of the no-allocation scratch failed: %s", cudaGetErrorString(e));
    return int(e);
  }
  *out = static_cast<double*>(p);
  return 0;
}

}  // namespace ss

// ===================================================================== C ABI ==
using namespace ss;

extern "C" {

int solve_matrix(double* a_matrix, double* b_matrix, int size, double* x_matrix, int nplasma) {
  int code = kSolveSingular;
  const int rc = run_single(kSolve, a_matrix, b_matrix, size, x_matrix, &code);
  if (rc) {
    // an engine failure leaves the caller's x untouched and reports the one
    // code whose caller action is "keep the old populations" (matrix_ion.c:287-291)
    fprintf(stderr, "solve_matrix: engine failure for plasma cell %d: %s\n", nplasma, g_last_error.c_str());
    return kSolveSingular;
  }
  return code;
}

int invert_matrix(double* matrix, double* inverted_matrix, int num_rows) {
  int code = kInvertSingular;
  const int rc = run_single(kInvert, matrix, nullptr, num_rows, inverted_matrix, &code);
  if (rc) {
    fprintf(stderr, "invert_matrix: engine failure: %s\n", g_last_error.c_str());
    return rc == int(cudaErrorMemoryAllocation) ? 8 /* GSL_ENOMEM */ : kInvertSingular;
  }
  return code;
}

const char* get_matrix_error_string(int error_code) {
  // the wording of the reference's GSL build (matrix_cpu.c:59-72)
  switch (error_code) {
    case 2: return "some matrix rows failing relative error check";
    case 3: return "some matrix rows failing absolute error check";
    case 4: return "Unsolvable matrix! Determinant is zero. Defaulting to no change";
    default: return "bad return from solve_matrix";
  }
}

int cusolver_create(void) { return ctx()->init(); }

int cusolver_destroy(void) {
  if (g_ctx) g_ctx->release();
  return 0;
}

const char* cusolver_get_error_string(int error) {
  switch (error) {
    case 0: return "The operation completed successfully";
    case 1: return "The matrix is singular";
    case 2: return "Some matrix rows fail the relative residual check";
    case 3: return "Some matrix rows fail the absolute residual check";
    case 4: return "Unsolvable matrix: a pivot is exactly zero";
    case 8: return "Device memory allocation failed";
    default: return "There was an unknown failure";
  }
}

int gpu_solve_matrix(double* a_matrix, double* b_vector, int size, double* x_vector) {
  return solve_matrix(a_matrix, b_vector, size, x_vector, -1);
}

int gpu_invert_matrix(double* matrix, double* inverse, int num_rows) {
  return invert_matrix(matrix, inverse, num_rows);
}

int solve_matrix_batched(int nsys, const int* n, const int64_t* offA, const double* A, const int64_t* offv,
                         const double* b, double* x, int* status) {
  return run_batched(kSolve, nsys, n, offA, A, offv, b, x, status, ctx()->mode);
}

int invert_matrix_batched(int nsys, const int* n, const int64_t* offA, const double* A, double* Ainv,
                          int* status) {
  return run_batched(kInvert, nsys, n, offA, A, nullptr, nullptr, Ainv, status, ctx()->mode);
}

int sirocco_set_precision(int mode) {
  if (mode != SIROCCO_FP64 && mode != SIROCCO_MIXED && mode != SIROCCO_FAST) {
    set_error("unknown precision mode %d", mode);
    return SIROCCO_EMODE;
  }
  ctx()->mode = mode;
  return 0;
}

int sirocco_plan_create(sirocco_plan** plan, int kind, int nsys, const int* n, const int64_t* offA,
                        const int64_t* offv, int mode) {
  if (!plan) {
    set_error("null plan pointer");
    return SIROCCO_EINVAL;
  }
  return plan_build(plan, kind, nsys, n, offA, offv, mode);
}

int sirocco_plan_execute(sirocco_plan* plan, const double* A, const double* b, double* out, int* status,
                         int* diag, void* stream) {
  if (!plan || (plan->nsys > 0 && (!A || !out || !status || (plan->kind == kSolve && !b)))) {
    set_error("invalid execute arguments");
    return SIROCCO_EINVAL;
  }
  return plan_run(plan, A, b, out, status, diag, static_cast<cudaStream_t>(stream));
}

int sirocco_plan_launches(const sirocco_plan* plan) { return plan ? int(plan->buckets.size()) : 0; }

int sirocco_plan_destroy(sirocco_plan* plan) {
  plan_free(plan);
  return 0;
}

const char* sirocco_last_error(void) { return g_last_error.c_str(); }

int matom_matrices_batched(int nsys, const int* n, const int64_t* offA, const int64_t* offv, const double* N,
                           const double* R, double* B, double* C, int* status) {
  return ss::run_matom(nsys, n, offA, offv, N, R, B, C, status);
}

int matom_sample_batched(int nq, int nsys, const int* n, const int64_t* offA, const double* C, const int* sys,
                         const int* level, const double* z, int* target) {
  return ss::run_matom_sample(nq, nsys, n, offA, C, sys, level, z, target);
}

int ion_populations_lockstep(int ncell, int nions, int nelem, const int* elem_first, const int* elem_n,
                             const int* istate, int h_elem, const double* elem_dens, double* ne, double* den,
                             sirocco_ion_assemble_fn assemble, void* user, int* status, int* iters) {
  return ss::run_ion_lockstep(ncell, nions, nelem, elem_first, elem_n, istate, h_elem, elem_dens, ne, den, assemble,
                              user, status, iters);
}

int matom_rate_matrices_batched(const sirocco_matom_table* tab, int ncell, const sirocco_matom_rates* rates, double* N,
                                double* R) {
  return ss::run_matom_rate_matrices(tab, ncell, rates, N, R);
}

int ion_rate_matrices_batched(const sirocco_ion_table* tab, int ncell, const sirocco_ion_rates* rates, const double* ne,
                              const double* nh1, const double* nh2, double* A, double* b) {
  return ss::run_ion_rate_matrices(tab, ncell, rates, ne, nh1, nh2, A, b);
}

int ion_populations_lockstep_rates(const sirocco_ion_table* tab, int ncell, const sirocco_ion_rates* rates, int h_elem,
                                   const double* elem_dens, double* ne, double* den, int* status, int* iters) {
  return ss::run_ion_lockstep_rates(tab, ncell, rates, h_elem, elem_dens, ne, den, status, iters);
}

int macro_pops_lockstep(int ncell, int n, int nion, const int* ion_first, const int* ion_nlte, const double* g,
                        const unsigned char* radiative, const double* scale, sirocco_macro_assemble_fn assemble,
                        void* user, double* pop, int* status, int* iters) {
  return ss::run_macro_pops(ncell, n, nion, ion_first, ion_nlte, g, radiative, scale, assemble, user, pop, status,
                            iters);
}

int solve_matrix_batched_noalloc(int nsys, int nmax, const int* n, const int64_t* offA, const double* A,
                                 const int64_t* offv, const double* b, double* x, int* status, void* stream) {
  if (nsys == 0) return 0;
  if (nsys < 0 || !n || !offA || !A || !offv || !b || !x || !status) {
    set_error("invalid arguments to solve_matrix_batched_noalloc");
    return SIROCCO_EINVAL;
  }
  if (nmax < 1 || nmax > kNoAllocMaxN) {
    set_error("solve_matrix_batched_noalloc: largest order %d outside 1..%d, the size of its static scratch",
              nmax, kNoAllocMaxN);
    return SIROCCO_ESIZE;
  }
  static_assert(global_panel_width(kNoAllocMaxN) == 16, "no-allocation path uses the 16-wide panel");
  const void* fn = reinterpret_cast<const void*>(&global_exact_kernel<kSolve, 16, true>);
  double* scratch = nullptr;
  int rc = noalloc_scratch(&scratch, fn);
  if (rc) return rc;
  const size_t smem = global_smem_bytes(nmax);
  BatchView v;
  v.n = n;
  v.offA = offA;
  v.offv = offv;
  v.A = A;
  v.b = b;
  v.out = x;
  v.status = status;
  v.diag = nullptr;
  v.list = nullptr;
  v.count = nsys;
  int64_t slab = int64_t(nmax) * nmax;
  // every CTA works in its own slab: no more CTAs than slabs of this size fit
  const int grid = int(std::min<int64_t>(std::min<int64_t>(nsys, 1024), int64_t(kNoAllocSlabs) * kNoAllocSlab / slab));
  void* args[] = {&v, &nmax, &scratch, &slab};
  SS_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(kGThreads), args, smem, static_cast<cudaStream_t>(stream)));
  return 0;
}

}  // extern "C"
