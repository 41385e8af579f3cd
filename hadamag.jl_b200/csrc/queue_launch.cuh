// queue_launch.cuh -- host launcher of the persistent queue sweep (sweep_queue.cuh),
// instantiated per precision in queue_fp64.cu / queue_fp32.cu.
#pragma once
#include "hm_ctx.h"
#include "sweep_queue.cuh"

namespace hm {

// Launch k_sre_queue<T, QS> with `blocks` CTAs on the context stream (inside the caller's
// graph capture).  Returns the warps launched.
template <typename T, int QS>
int launch_queue_kernel(hm_ctx *c, const QArgs &a, int ctas_per_sm, long long total_units, int *nwarps) {
  using V = typename VT<T>::V;
  const size_t smem = (size_t)QWARPS * 32 * 32 * sizeof(V);
  auto kern = k_sre_queue<T, QS>;
  HM_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, QWARPS * 32, smem));
  if (occ < 1) occ = 1;
  if (ctas_per_sm > 0 && ctas_per_sm < occ) occ = ctas_per_sm;
  long long blocks = (long long)c->num_sms * occ;
  const long long need = (total_units + QWARPS - 1) / QWARPS;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  kern<<<(unsigned)blocks, QWARPS * 32, smem, c->stream>>>(a);
  HM_CUDA(c, cudaGetLastError());
  *nwarps = (int)blocks * QWARPS;
  return HM_OK;
}

// warps the launch will use (for sizing the slots before the launch)
template <typename T, int QS>
int queue_warps(hm_ctx *c, int ctas_per_sm, long long total_units, int *nwarps) {
  using V = typename VT<T>::V;
  const size_t smem = (size_t)QWARPS * 32 * 32 * sizeof(V);
  auto kern = k_sre_queue<T, QS>;
  HM_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, QWARPS * 32, smem));
  if (occ < 1) occ = 1;
  if (ctas_per_sm > 0 && ctas_per_sm < occ) occ = ctas_per_sm;
  long long blocks = (long long)c->num_sms * occ;
  const long long need = (total_units + QWARPS - 1) / QWARPS;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  *nwarps = (int)blocks * QWARPS;
  return HM_OK;
}

}  // namespace hm
