// sre_launch.cuh -- host launchers for the exact-SRE kernels (instantiated per precision
// in sre_fp64.cu / sre_fp32.cu).
#pragma once
#include "hm_ctx.h"
#include "sre_kernels.cuh"

namespace hm {

// Tunables of the two-pass sweep: X-strings per batch and ring slots.  X * S * 2^(n-1)
// complex values are live in the ring; at n = 20 (FP64) X = 2, S = 3 is 48 MiB, which
// stays resident in the 126 MB L2 next to the 16 MiB state.
struct TwoPassCfg {
  int X = 2;
  int X_set = 0;  // X was set explicitly (otherwise 2 for FP64, 4 for FP32)
  int S = 3;
  int upw = 1;  // warp units per warp per CTA item
  int fence_all = 0;  // every lane fences its own stores before the completion signal
  int release = 0;    // completion signal: 0 fence.sc + atomic, 1 red.release, 2 fence.acq_rel + atomic
  int stage_b = 0;    // pass 1 stages the partner row through shared memory (cp.async)
};

TwoPassCfg &twopass_cfg();

template <typename T, int R, int NB, int QS>
static int launch_fused(hm_ctx *c, const SreArgs &a0, int *nwarps_out) {
  using V = typename VT<T>::V;
  SreArgs a = a0;
  constexpr int PB = ilog2c(R) + 5;
  const size_t smem = (size_t)FUSED_WARPS * 32 * R * sizeof(V);
  auto kern = k_sre_fused<T, R, NB, QS>;
  HM_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, FUSED_WARPS * 32, smem));
  if (occ < 1) occ = 1;
  const uint64_t XPW = 1ull << (PB - NB);
  const uint64_t ngroups = (a.k_end - a.k_begin + XPW - 1) / XPW;
  uint64_t blocks = (ngroups + FUSED_WARPS - 1) / FUSED_WARPS;
  const uint64_t maxb = (uint64_t)c->num_sms * occ;
  if (blocks > maxb) blocks = maxb;
  if (blocks < 1) blocks = 1;
  const int nwarps = (int)blocks * FUSED_WARPS;
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap,
                    sizeof(double) * 2 * (QSet<QS>::NQ + 1) * (size_t)nwarps));
  a.partials = c->d_partials;
  kern<<<(unsigned)blocks, FUSED_WARPS * 32, smem, c->stream>>>(a);
  HM_CUDA(c, cudaGetLastError());
  *nwarps_out = nwarps;
  return HM_OK;
}

template <typename T, int R, int HI, int QS>
static int launch_2pass(hm_ctx *c, const SreArgs &a0, int *nwarps_out) {
  using V = typename VT<T>::V;
  SreArgs a = a0;
  const TwoPassCfg cfg = twopass_cfg();
  const size_t smem = (size_t)SRE_WARPS * 32 * R * sizeof(V);
  auto kern = k_sre_2pass<T, R, HI, QS>;
  HM_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, SRE_WARPS * 32, smem));
  if (occ < 1) occ = 1;
  // FP32 rows are half the bytes: twice the X-strings per batch fit the same L2 budget
  a.X = cfg.X_set ? cfg.X : (sizeof(T) == 8 ? 2 : 4);
  a.S = cfg.S;
  a.flags = (cfg.fence_all ? 2 : 0) | (cfg.release == 1 ? 4 : 0) | (cfg.release == 2 ? 8 : 0) | (cfg.stage_b ? 16 : 0);
  const uint64_t len = a.k_end - a.k_begin;
  a.nbatch = (int)((len + a.X - 1) / a.X);
  const uint64_t U = 1ull << HI;
  a.upw = cfg.upw;
  while (a.upw > 1 && (uint64_t)a.X * U < (uint64_t)SRE_WARPS * a.upw) a.upw >>= 1;
  const long long K = (long long)((a.X * U) / (SRE_WARPS * a.upw));  // CTA items per pass per batch
  a.nitems = 2 * K * (long long)a.nbatch;
  const size_t inter_bytes = (size_t)a.S * a.X * ((size_t)1 << (a.n - 1)) * sizeof(V);
  HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, inter_bytes));
  a.inter = c->d_inter;
  const size_t ctrl_words = 8 + 2 * (size_t)a.S;
  HM_TRY(ensure_dev(c, (void **)&c->d_ctrl, &c->ctrl_cap, ctrl_words * sizeof(unsigned)));
  HM_CUDA(c, cudaMemsetAsync(c->d_ctrl, 0, ctrl_words * sizeof(unsigned), c->stream));
  a.ctrl = c->d_ctrl;
  // bit-swapped copies of psi for the X-strings 1 <= x < 2^PB (Gray indices below 2^PB)
  constexpr int PB = ilog2c(R) + 5;
  if (a.k_begin < (1ull << PB)) {
    const size_t len = (size_t)1 << a.n;
    HM_TRY(ensure_dev(c, &c->d_aux2, &c->aux2_cap, (size_t)PB * len * sizeof(V)));
    k_psi_swapped<V><<<c->num_sms * 8, 256, 0, c->stream>>>(reinterpret_cast<const V *>(a.psi),
                                                            reinterpret_cast<V *>(c->d_aux2), a.n, PB);
    HM_CUDA(c, cudaGetLastError());
    for (int j = 0; j < PB; ++j) a.psi_sw[j] = reinterpret_cast<const V *>(c->d_aux2) + (size_t)j * len;
  }
  int blocks = c->num_sms * occ;
  if ((long long)blocks > a.nitems) blocks = (int)a.nitems;
  if (blocks < 1) blocks = 1;
  const int nwarps = blocks * SRE_WARPS;
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap,
                    sizeof(double) * 2 * (QSet<QS>::NQ + 1) * (size_t)nwarps));
  a.partials = c->d_partials;
  kern<<<blocks, SRE_WARPS * 32, smem, c->stream>>>(a);
  HM_CUDA(c, cudaGetLastError());
  *nwarps_out = nwarps;
  return HM_OK;
}

#define HM_FUSED_CASE(NBv)                                         \
  case NBv:                                                        \
    return launch_fused<T, R, ((NBv) <= PB ? (NBv) : PB), QS>(c, a, nw);
#define HM_2P_CASE(HIv)                                            \
  case HIv:                                                        \
    return launch_2pass<T, R, ((HIv) <= PB ? (HIv) : PB), QS>(c, a, nw);

template <typename T, int R, int QS>
static int dispatch_sre(hm_ctx *c, const SreArgs &a, int *nw) {
  constexpr int PB = ilog2c(R) + 5;
  const int nb = a.n - 1;
  if (nb <= PB) {
    switch (nb) {
      HM_FUSED_CASE(0)
      HM_FUSED_CASE(1)
      HM_FUSED_CASE(2)
      HM_FUSED_CASE(3)
      HM_FUSED_CASE(4)
      HM_FUSED_CASE(5)
      HM_FUSED_CASE(6)
      HM_FUSED_CASE(7)
      HM_FUSED_CASE(8)
      HM_FUSED_CASE(9)
      HM_FUSED_CASE(10)
      HM_FUSED_CASE(11)
      default:
        break;
    }
  } else {
    switch (nb - PB) {
      HM_2P_CASE(1)
      HM_2P_CASE(2)
      HM_2P_CASE(3)
      HM_2P_CASE(4)
      HM_2P_CASE(5)
      HM_2P_CASE(6)
      HM_2P_CASE(7)
      HM_2P_CASE(8)
      HM_2P_CASE(9)
      HM_2P_CASE(10)
      HM_2P_CASE(11)
      default:
        break;
    }
  }
  return set_err(c, HM_ERR_SIZE, "n = %d outside the fused range of this precision", a.n);
}

// one precision and moment set; returns the number of per-warp partial records written
template <typename T, int R, int QS>
int launch_sre_qs(hm_ctx *c, const void *psi_dev, int n, uint64_t kb, uint64_t ke, const QParams &qp,
                  int *nwarps) {
  SreArgs a;
  memset(&a, 0, sizeof a);
  a.psi = psi_dev;
  a.n = n;
  a.k_begin = kb;
  a.k_end = ke;
  a.qp = qp;
  a.spin_limit = 1ll << 34;
  return dispatch_sre<T, R, QS>(c, a, nwarps);
}

}  // namespace hm
