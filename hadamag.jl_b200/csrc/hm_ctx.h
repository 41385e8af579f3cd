// hm_ctx.h -- host-side context shared by the C-ABI and the launchers (not part of the ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <string>

#include "../../include/hadamag_b200.h"

struct hm_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  long long launches = 0;  // kernels launched by the current / last call
  std::string err;

  // grow-only device buffers
  void *d_psi = nullptr;  // double2 copy of the input state
  size_t psi_cap = 0;
  void *d_psi32 = nullptr;  // float2 copy (FP32 path)
  size_t psi32_cap = 0;
  void *d_inter = nullptr;  // two-pass ring / plain-path column batch
  size_t inter_cap = 0;
  double *d_partials = nullptr;
  size_t partials_cap = 0;
  unsigned *d_ctrl = nullptr;  // stage index of the two-pass stage kernels
  size_t ctrl_cap = 0;
  double *d_out = nullptr;  // fold output
  size_t out_cap = 0;
  void *d_aux = nullptr;  // per-feature scratch (masks, Mana, MC state)
  size_t aux_cap = 0;
  void *d_aux2 = nullptr;
  size_t aux2_cap = 0;
  double *h_out = nullptr;  // pinned host mirror of d_out
  size_t h_out_cap = 0;
  void *h_pin = nullptr;  // pinned host scratch
  size_t h_pin_cap = 0;
  void *d_queue = nullptr;  // queue sweep: state table, batch counters, per-warp slots
  size_t queue_cap = 0;
};

namespace hm {

// error helpers: record the message on the context and return the status
inline int set_err(hm_ctx *c, int code, const char *fmt, ...) __attribute__((format(printf, 3, 4)));
inline int set_err(hm_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

// On failure the runtime's error state is cleared (cudaGetLastError) so that a non-sticky
// error is reported once, by the call that hit it, and not again by the next call's checks.
#define HM_CUDA(c, call)                                                                              \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) {                                                                          \
      cudaGetLastError();                                                                             \
      return ::hm::set_err((c), HM_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                           __FILE__, __LINE__);                                                       \
    }                                                                                                 \
  } while (0)

#define HM_TRY(expr)          \
  do {                        \
    int rc_ = (expr);         \
    if (rc_ != HM_OK) return rc_; \
  } while (0)

// grow-only device buffer
inline int ensure_dev(hm_ctx *c, void **p, size_t *cap, size_t bytes) {
  if (bytes <= *cap && *p) return HM_OK;
  if (*p) {
    cudaStreamSynchronize(c->stream);
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
  }
  size_t want = bytes < 256 ? 256 : bytes;
  cudaError_t e = cudaMalloc(p, want);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_err(c, HM_ERR_OOM, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
  }
  *cap = want;
  return HM_OK;
}

inline int ensure_host(hm_ctx *c, void **p, size_t *cap, size_t bytes) {
  if (bytes <= *cap && *p) return HM_OK;
  if (*p) {
    cudaStreamSynchronize(c->stream);
    cudaFreeHost(*p);
    *p = nullptr;
    *cap = 0;
  }
  size_t want = bytes < 256 ? 256 : bytes;
  cudaError_t e = cudaMallocHost(p, want);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_err(c, HM_ERR_OOM, "cudaMallocHost(%zu) failed: %s", want, cudaGetErrorString(e));
  }
  *cap = want;
  return HM_OK;
}

struct QReq {
  double q[4];
  int nq;
};

// One state of a queue sweep: a device-resident double2 state and a Gray range.
struct QueueItem {
  const double2 *psi;
  int n;
  uint64_t kb, ke;
};

// Tunables of the queue sweep (hm_set_param / hm_autotune): X-strings per ring slot of
// the largest two-pass state (X, when set; else the tuned table; else a slot of
// slot_mib MiB), K ring slots, units claimed per atomic, CTAs per SM (0: occupancy).
struct QueueCfg {
  int X = 0;
  int X_set = 0;
  int slot_mib = 16;
  int K = 4;
  int chunk = 1;
  int ctas_per_sm = 0;
  int engine = 0;  // single-state sweeps: 0 automatic, 1 stage kernels, 2 queue sweep
  int stall_test = 0;  // test of the bounded waits (HM_PARAM_QUEUE_STALL_TEST)
  int lead = 2;        // batches between a batch's pass 1 and pass 2 (HM_PARAM_QUEUE_LEAD)
  int batch_split_n = 15;  // hm_sre_batched: states from this n up run one per call (HM_PARAM_BATCH_SPLIT_N)
  int tuned_x[2][32] = {};
  int tuned_cps[2][32] = {};
  int tuned_engine[2][32] = {};  // hm_autotune's choice per (precision, n): 0 none, 1 stage, 2 queue
};
QueueCfg &queue_cfg();
int sweep_engine(int n, int precision);

// Exact-SRE raw sums of several states in one persistent launch (12 <= n <= 21 two-pass
// states and n <= 11 one-warp states); out_dd per item: [p2_hi, p2_lo, m0_hi, m0_lo, ...].
int run_queue(hm_ctx *c, const QueueItem *items, int nitems, const QReq &q, int precision, double *out_dd);
// as run_queue, with FP32's x = 0 transforms split off into an FP64 launch
int run_queue_sre(hm_ctx *c, const QueueItem *items, int nitems, const QReq &q, int precision, double *out_dd);

// exact SRE raw sums over Gray indices [kb, ke) of a device-resident double2 state.
// out_dd (host): [p2_hi, p2_lo, m0_hi, m0_lo, ...] for each requested q.
int run_sre(hm_ctx *c, const double2 *psi_dev, int n, uint64_t kb, uint64_t ke, const QReq &q, int precision,
            double *out_dd);
int run_sre_plain(hm_ctx *c, const double2 *psi_dev, int n, uint64_t kb, uint64_t ke, const QReq &q,
                  double *out_dd);

}  // namespace hm
