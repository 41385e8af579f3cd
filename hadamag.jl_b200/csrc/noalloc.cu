// noalloc.cu -- exact SRE for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code running inside another framework's
// allocator-controlled region, plugins that must not grow the process's device footprint
// after start-up, or hosts whose device memory is fully reserved by a pool they do not
// own.  hm_sre_noalloc serves them with the fused single-warp exact-SRE kernel (n <= 11)
// and a scratch area that lives in this file as a statically sized device array: the
// copy of the state, the per-warp partial sums and the folded result.  Every GPU that
// loads the library keeps that array until the process exits.
#include <math.h>

#include <mutex>

#include "../../include/hadamag_b200.h"
#include "sre_kernels.cuh"

namespace {

constexpr int NOALLOC_MAX_N = HM_NOALLOC_MAX_N;    // fused path: n - 1 <= 10 element bits
constexpr int NOALLOC_STATE = 1 << NOALLOC_MAX_N;  // double2 state slots
// A fixed cap on the per-warp partial records, independent of the device: the grid is
// clamped to NOALLOC_WARPS / FUSED_WARPS blocks whatever the SM count.  (4736 warps is
// 148 SMs x 8 CTAs on a B200; on other devices the cap only changes how many X-string
// groups each warp loops over, never the result.)
constexpr int NOALLOC_WARPS = 148 * 8 * hm::FUSED_WARPS;
constexpr int NOALLOC_NSUM = 5;                    // p2 + up to four moments
constexpr int NOALLOC_DOUBLES = 2 * NOALLOC_STATE + 2 * NOALLOC_NSUM * NOALLOC_WARPS + 2 * NOALLOC_NSUM;

// the scratch: [state (2^11 double2)] [per-warp double-double partials] [fold output]
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

// In host code g_noalloc_scratch names a host-side stand-in, not device memory: its
// device address is looked up with the device current and cached per device, together
// with the context it belongs to.  A device reset (cudaDeviceReset) or a destroyed and
// recreated primary context reloads the module at another address, so the address is
// looked up again whenever the device's current context is not the cached one.
typedef int (*CtxGetCurrentFn)(void **);  // cuCtxGetCurrent (CUresult, CUcontext *)
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[64] = {nullptr};
void *g_noalloc_ctx[64] = {nullptr};

CtxGetCurrentFn ctx_get_current() {
  static std::once_flag once;
  static CtxGetCurrentFn fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

int noalloc_scratch(int dev, double **out) {
  if (dev < 0 || dev >= 64) return HM_ERR_CUDA;
  CtxGetCurrentFn get = ctx_get_current();
  if (!get) return HM_ERR_CUDA;
  void *cur = nullptr;  // null when no context is bound to this thread yet
  if (get(&cur) != 0) return HM_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev] || cur == nullptr || g_noalloc_ctx[dev] != cur) {
    // the lookup binds the device's primary context to the thread when none is bound
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      g_noalloc_ptr[dev] = nullptr;
      return HM_ERR_CUDA;
    }
    if (get(&cur) != 0 || cur == nullptr) return HM_ERR_CUDA;
    g_noalloc_ptr[dev] = static_cast<double *>(p);
    g_noalloc_ctx[dev] = cur;
  }
  *out = g_noalloc_ptr[dev];
  return HM_OK;
}

template <int QS>
int noalloc_launch(int n, const double2 *psi, double *partials, hm::QParams qp, cudaStream_t st, int *nwarps) {
  hm::SreArgs a;
  memset(&a, 0, sizeof a);
  a.psi = psi;
  a.n = n;
  a.k_begin = 0;
  a.k_end = 1ull << n;
  a.qp = qp;
  a.partials = partials;
  const int PB = 10, nb = n - 1;
  const uint64_t xpw = 1ull << (PB - nb);
  const uint64_t ngroups = (a.k_end + xpw - 1) / xpw;
  int blocks = (int)((ngroups + hm::FUSED_WARPS - 1) / hm::FUSED_WARPS);
  if (blocks > NOALLOC_WARPS / hm::FUSED_WARPS) blocks = NOALLOC_WARPS / hm::FUSED_WARPS;
  const size_t smem = (size_t)hm::FUSED_WARPS * 32 * 32 * sizeof(double2);
#define HM_NOALLOC_CASE(NBv)                                                                            \
  case NBv:                                                                                             \
    if (cudaFuncSetAttribute(hm::k_sre_fused<double, 32, NBv, QS>,                                      \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)    \
      return HM_ERR_CUDA;                                                                               \
    hm::k_sre_fused<double, 32, NBv, QS><<<blocks, hm::FUSED_WARPS * 32, smem, st>>>(a);               \
    break;
  switch (nb) {
    HM_NOALLOC_CASE(0)
    HM_NOALLOC_CASE(1)
    HM_NOALLOC_CASE(2)
    HM_NOALLOC_CASE(3)
    HM_NOALLOC_CASE(4)
    HM_NOALLOC_CASE(5)
    HM_NOALLOC_CASE(6)
    HM_NOALLOC_CASE(7)
    HM_NOALLOC_CASE(8)
    HM_NOALLOC_CASE(9)
    HM_NOALLOC_CASE(10)
    default:
      return HM_ERR_SIZE;
  }
#undef HM_NOALLOC_CASE
  *nwarps = blocks * hm::FUSED_WARPS;
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

}  // namespace

// See include/hadamag_b200.h.
extern "C" int hm_sre_noalloc(const double *psi, int n, const double *qs, int nq, double *out_sre,
                              double *out_lost, void *cuda_stream) {
  if (!psi || !qs || !out_sre || !out_lost) return HM_ERR_ARG;
  if (n < 1 || n > NOALLOC_MAX_N) return HM_ERR_SIZE;
  if (nq < 1 || nq > 4) return HM_ERR_ARG;
  for (int i = 0; i < nq; ++i)
    if (!(qs[i] >= 1.0 && qs[i] <= 16.0)) return HM_ERR_Q;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return HM_ERR_CUDA;
  double *scratch = nullptr;
  const int rc0 = noalloc_scratch(dev, &scratch);
  if (rc0 != HM_OK) return rc0;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  double2 *state = reinterpret_cast<double2 *>(scratch);
  double *partials = scratch + 2 * NOALLOC_STATE;
  double *folded = partials + 2 * NOALLOC_NSUM * NOALLOC_WARPS;
  const size_t len = (size_t)1 << n;
  if (cudaMemcpyAsync(state, psi, len * sizeof(double2), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return HM_ERR_CUDA;
  // the moment set, as the allocating path chooses it: q = 2 only, q in {2, 3}, or generic
  hm::QParams qp;
  memset(&qp, 0, sizeof qp);
  int idx[4], kind;
  bool only23 = true, has3 = false;
  for (int i = 0; i < nq; ++i) {
    if (qs[i] != 2.0 && qs[i] != 3.0) only23 = false;
    if (qs[i] == 3.0) has3 = true;
  }
  if (only23 && !has3) {
    kind = hm::QS_Q2;
    for (int i = 0; i < nq; ++i) idx[i] = 1;
  } else if (only23) {
    kind = hm::QS_Q23;
    for (int i = 0; i < nq; ++i) idx[i] = qs[i] == 2.0 ? 1 : 2;
  } else {
    kind = hm::QS_GEN;
    qp.nq = nq;
    for (int i = 0; i < 4; ++i) qp.q[i] = i < nq ? qs[i] : 2.0;
    for (int i = 0; i < nq; ++i) idx[i] = 1 + i;
  }
  const int nsum = 1 + (kind == hm::QS_Q2 ? 1 : (kind == hm::QS_Q23 ? 2 : 4));
  // every warp of the fused kernel overwrites its own partial record and the fold
  // overwrites its output, so nothing left by the previous call needs clearing
  int nwarps = 0, rc = HM_OK;
  if (kind == hm::QS_Q2)
    rc = noalloc_launch<hm::QS_Q2>(n, state, partials, qp, st, &nwarps);
  else if (kind == hm::QS_Q23)
    rc = noalloc_launch<hm::QS_Q23>(n, state, partials, qp, st, &nwarps);
  else
    rc = noalloc_launch<hm::QS_GEN>(n, state, partials, qp, st, &nwarps);
  if (rc != HM_OK) return rc;
  hm::k_fold_partials<<<1, 256, 0, st>>>(partials, nwarps, nsum, folded);
  if (cudaGetLastError() != cudaSuccess) return HM_ERR_CUDA;
  double h[2 * NOALLOC_NSUM];
  if (cudaMemcpyAsync(h, folded, sizeof(double) * 2 * nsum, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return HM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return HM_ERR_CUDA;
  const double dim = ldexp(1.0, n);
  for (int i = 0; i < nq; ++i) out_sre[i] = -log2((h[2 * idx[i]] + h[2 * idx[i] + 1]) / dim);
  *out_lost = fabs(1.0 - (h[0] + h[1]) / dim);
  return HM_OK;
}
