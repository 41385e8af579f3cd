// sre_host.cu -- exact-SRE driver: precision dispatch, fold of the per-warp partials,
// result read-back.
#include <cudaTypedefs.h>
#include <math.h>

#include <mutex>
#include <vector>

#include "sre_launch.cuh"

namespace hm {

template <typename T, int R, int QS>
int launch_sre_qs(hm_ctx *c, const void *psi_dev, int n, uint64_t kb, uint64_t ke, const QParams &qp, int *nwarps);

template <typename T>
static int launch_sre_prec(hm_ctx *c, const void *psi_dev, int n, uint64_t kb, uint64_t ke, int kind,
                           const QParams &qp, int *nwarps) {
  switch (kind) {
    case QS_Q2:
      return launch_sre_qs<T, 32, QS_Q2>(c, psi_dev, n, kb, ke, qp, nwarps);
    case QS_Q23:
      return launch_sre_qs<T, 32, QS_Q23>(c, psi_dev, n, kb, ke, qp, nwarps);
    default:
      return launch_sre_qs<T, 32, QS_GEN>(c, psi_dev, n, kb, ke, qp, nwarps);
  }
}

TwoPassCfg &twopass_cfg() {
  static TwoPassCfg cfg;
  return cfg;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link-time
// dependency on libcuda), looked up once per process.
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

bool encode_ring_tmap(CUtensorMap *m, void *ring, int scalar_bytes, int C, int U, int T, int two_x,
                      uint64_t x_stride_bytes, const TmaGeom &g) {
  // innermost box extent and every stride must be multiples of 16 bytes; boxes <= 256
  const uint64_t row_bytes = (uint64_t)2 * C * scalar_bytes;
  if ((g.box0 * scalar_bytes) % 16 != 0 || row_bytes % 16 != 0 || g.box0 > 256 || g.box2 > 256) return false;
  if (g.nb0 * g.box0 != 2 * C || g.nb2 * g.box2 != T) return false;
  if (((uintptr_t)ring & 15) != 0) return false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)2 * C, (cuuint64_t)U, (cuuint64_t)T, (cuuint64_t)two_x};
  const cuuint64_t strides[3] = {row_bytes, row_bytes * (uint64_t)U, x_stride_bytes};
  const cuuint32_t box[4] = {(cuuint32_t)g.box0, 1u, (cuuint32_t)g.box2, 1u};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  const CUresult r =
      enc(m, scalar_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ring, dims,
          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

__global__ void k_stage_advance(unsigned *stage, unsigned count) { stage[0] += count; }

__global__ void k_fold_partials(const double *__restrict__ partials, int nwarps, int nsum, double *out) {
  // one block; thread t folds warps t, t + blockDim, ... then a fixed-shape tree
  __shared__ dd sh[256][5];
  const int t = threadIdx.x;
  dd acc[5];
  for (int s = 0; s < 5; ++s) acc[s] = dd{0.0, 0.0};
  for (int w = t; w < nwarps; w += blockDim.x)
    for (int s = 0; s < nsum; ++s) {
      dd v{partials[(size_t)w * 2 * nsum + 2 * s], partials[(size_t)w * 2 * nsum + 2 * s + 1]};
      dd_add_dd(acc[s], v);
    }
  for (int s = 0; s < 5; ++s) sh[t][s] = acc[s];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (t < o)
      for (int s = 0; s < nsum; ++s) dd_add_dd(sh[t][s], sh[t + o][s]);
    __syncthreads();
  }
  if (t == 0)
    for (int s = 0; s < nsum; ++s) {
      out[2 * s] = sh[0][s].hi;
      out[2 * s + 1] = sh[0][s].lo;
    }
}

__global__ void k_psi_to_f32(const double2 *__restrict__ in, float2 *__restrict__ out, uint64_t len) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 v = in[i];
    out[i] = make_float2((float)v.x, (float)v.y);
  }
}

// (hi, lo) += (b_hi, b_lo), Knuth TwoSum on the high parts
static void dd_add_host(double *a, double bh, double bl) {
  const double s = a[0] + bh;
  const double bb = s - a[0];
  const double err = (a[0] - (s - bb)) + (bh - bb);
  const double lo = a[1] + bl + err;
  a[0] = s + lo;
  a[1] = lo - (a[0] - s);
}

// Map requested q values onto a kernel moment set.  Returns the kind and, per request,
// the index of its sum in the kernel output (1-based; 0 is sum F^2).
static int choose_qs(const QReq &q, QParams &qp, int *idx) {
  bool only23 = true, has3 = false;
  for (int i = 0; i < q.nq; ++i) {
    if (q.q[i] != 2.0 && q.q[i] != 3.0) only23 = false;
    if (q.q[i] == 3.0) has3 = true;
  }
  memset(&qp, 0, sizeof qp);
  if (only23 && !has3) {
    for (int i = 0; i < q.nq; ++i) idx[i] = 1;
    return QS_Q2;
  }
  if (only23) {
    for (int i = 0; i < q.nq; ++i) idx[i] = q.q[i] == 2.0 ? 1 : 2;
    return QS_Q23;
  }
  qp.nq = q.nq;
  for (int i = 0; i < q.nq; ++i) {
    qp.q[i] = q.q[i];
    idx[i] = 1 + i;
  }
  for (int i = q.nq; i < 4; ++i) qp.q[i] = 2.0;
  return QS_GEN;
}

int queue_choose_qs(const QReq &q, QParams &qp, int *idx) { return choose_qs(q, qp, idx); }

// Sweep of one state's two-pass sizes: 1 = stage kernels, 2 = queue sweep.  HM_PARAM_ENGINE
// forces one; otherwise the choice hm_autotune recorded for (n, precision), else the stage
// kernels (measured faster for a single large state on B200: 3.99 vs 4.8 us per X-string at
// n = 20 in FP64).
int sweep_engine(int n, int precision) {
  const QueueCfg &qc = queue_cfg();
  if (qc.engine == 1 || qc.engine == 2) return qc.engine;
  const int t = (n >= 0 && n < 32) ? qc.tuned_engine[precision == HM_FP32 ? 1 : 0][n] : 0;
  return t ? t : 1;
}

// Queue sweep of several states.  In FP32 the x = 0 transform of every state (F = WHT of
// |psi|^2, whose F(0)^4 = 1 can dominate m) runs in an FP64 launch of its own and is added
// as a double-double term, as on the stage-kernel path.
int run_queue_sre(hm_ctx *c, const QueueItem *items, int nitems, const QReq &q, int precision, double *out_dd) {
  const int w = 2 * (1 + q.nq);
  if (precision != HM_FP32) return run_queue(c, items, nitems, q, HM_FP64, out_dd);
  std::vector<QueueItem> zero, rest(items, items + nitems);
  std::vector<int> zidx;
  for (int i = 0; i < nitems; ++i)
    if (items[i].kb == 0 && items[i].ke > 0) {
      zero.push_back(QueueItem{items[i].psi, items[i].n, 0, 1});
      zidx.push_back(i);
      rest[i].kb = 1;
    }
  std::vector<double> zout(zero.size() * w);
  double ms0 = 0.0;
  if (!zero.empty()) {
    HM_TRY(run_queue(c, zero.data(), (int)zero.size(), q, HM_FP64, zout.data()));
    ms0 = c->last_ms;
  }
  HM_TRY(run_queue(c, rest.data(), nitems, q, HM_FP32, out_dd));
  c->last_ms += ms0;
  for (size_t z = 0; z < zero.size(); ++z)
    for (int t = 0; t < 1 + q.nq; ++t) dd_add_host(out_dd + (size_t)zidx[z] * w + 2 * t, zout[z * w + 2 * t],
                                                  zout[z * w + 2 * t + 1]);
  return HM_OK;
}

int run_sre(hm_ctx *c, const double2 *psi_dev, int n, uint64_t kb, uint64_t ke, const QReq &q, int precision,
            double *out_dd) {
  if (precision == HM_PLAIN || n > 24 || n < 1) return run_sre_plain(c, psi_dev, n, kb, ke, q, out_dd);
  if (ke <= kb) {
    for (int i = 0; i < 2 * (1 + q.nq); ++i) out_dd[i] = 0.0;
    return HM_OK;
  }
  if (n >= 12 && n <= 21 && sweep_engine(n, precision) == 2) {
    const QueueItem it{psi_dev, n, kb, ke};
    return run_queue_sre(c, &it, 1, q, precision, out_dd);
  }
  QParams qp;
  int idx[4];
  const int kind = choose_qs(q, qp, idx);
  const int nsum = 1 + (kind == QS_Q2 ? 1 : (kind == QS_Q23 ? 2 : 4));
  const uint64_t len = 1ull << n;
  // the fused kernels (n <= 11) read the FP64 state in both precisions; the FP32 two-pass
  // kernels read an FP32 copy
  const void *psi_k = psi_dev;
  if (precision == HM_FP32 && (n - 1) > 10) {
    HM_TRY(ensure_dev(c, &c->d_psi32, &c->psi32_cap, len * sizeof(float2)));
    k_psi_to_f32<<<c->num_sms * 4, 256, 0, c->stream>>>(psi_dev, (float2 *)c->d_psi32, len);
    c->launches += 1;
    HM_CUDA(c, cudaGetLastError());
    psi_k = c->d_psi32;
  }
  // x = 0 (F = WHT of |psi|^2, whose F(0)^4 = 1 can dominate m) always runs in FP64: the
  // FP64 kernels build it themselves (top-bit pairing in pass 1, scale 1), and an FP32 call
  // runs it as an FP64 call of its own, since the FP32 kernels would round it
  const bool split_zero = kb == 0 && precision == HM_FP32;
  const uint64_t kb_main = split_zero ? 1 : kb;
  int nwarps = 0;
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  if (kb_main >= ke) {
    // only x = 0 requested: the main kernels have nothing to do
    HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap, sizeof(double) * 16));
    HM_CUDA(c, cudaMemsetAsync(c->d_partials, 0, sizeof(double) * 2 * nsum, c->stream));
    nwarps = 1;
  } else if (precision == HM_FP32) {
    HM_TRY((launch_sre_prec<float>(c, psi_k, n, kb_main, ke, kind, qp, &nwarps)));
  } else {
    HM_TRY((launch_sre_prec<double>(c, psi_k, n, kb_main, ke, kind, qp, &nwarps)));
  }
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, sizeof(double) * 16));
  k_fold_partials<<<1, 256, 0, c->stream>>>(c->d_partials, nwarps, nsum, c->d_out);
  c->launches += 1;
  HM_CUDA(c, cudaGetLastError());
  HM_TRY(ensure_host(c, (void **)&c->h_out, &c->h_out_cap, sizeof(double) * 16 + 64));
  HM_CUDA(c, cudaMemcpyAsync(c->h_out, c->d_out, sizeof(double) * 2 * nsum, cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  out_dd[0] = c->h_out[0];
  out_dd[1] = c->h_out[1];
  for (int i = 0; i < q.nq; ++i) {
    out_dd[2 + 2 * i] = c->h_out[2 * idx[i]];
    out_dd[3 + 2 * i] = c->h_out[2 * idx[i] + 1];
  }
  if (split_zero) {
    // x = 0 (F = WHT of |psi|^2) is not part of the stage kernels' sweep: one FP64
    // transform of the queue sweep, added as a double-double term
    const double ms_main = c->last_ms;
    double z[10];
    HM_TRY(run_sre(c, psi_dev, n, 0, 1, q, HM_FP64, z));
    c->last_ms += ms_main;
    for (int t = 0; t < 1 + q.nq; ++t) dd_add_host(out_dd + 2 * t, z[2 * t], z[2 * t + 1]);
  }
  return HM_OK;
}

}  // namespace hm

// Fill psi with a unit-norm pattern state (values do not matter for timing).
static __global__ void k_tune_state(double2 *psi, uint64_t len) {
  const double s = rsqrt((double)len);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi((double)(i % 977) / 977.0 * 2.0, &sn, &cs);
    psi[i] = make_double2(s * cs, s * sn);
  }
}

// Autotuner of the two-pass sweep of one (n, precision): times hm_sre_range on `sample`
// Gray indices (starting at 1024, where the sweep's steady state begins) for
//   the stage kernels with X = 1, 2, 4, ... X-strings per stage (ring up to 1 GiB), and
//   the queue sweep with X = 1, 2, 4, ... X-strings per ring slot (4 slots up to 1 GiB)
//   at full occupancy and at one CTA per SM,
// keeps the fastest (kernel time, CUDA events) and records engine, batch size and CTAs per
// SM for this (n, precision); later calls use them unless a knob forces another choice.
extern "C" int hm_autotune(hm_ctx *c, int n, int precision, int *best_x, double *best_us_per_x) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!best_x || !best_us_per_x) return hm::set_err(c, HM_ERR_ARG, "null output pointer");
  if (n < 12 || n > 21) return hm::set_err(c, HM_ERR_SIZE, "autotune: n = %d outside the two-pass range [12, 21]", n);
  if (precision != HM_FP64 && precision != HM_FP32)
    return hm::set_err(c, HM_ERR_ARG, "autotune: precision must be HM_FP64 or HM_FP32");
  HM_CUDA(c, cudaSetDevice(c->device));
  const uint64_t len = 1ull << n;
  HM_TRY(hm::ensure_dev(c, &c->d_psi, &c->psi_cap, len * sizeof(double2)));
  k_tune_state<<<c->num_sms * 4, 256, 0, c->stream>>>((double2 *)c->d_psi, len);
  HM_CUDA(c, cudaGetLastError());
  hm::TwoPassCfg &cfg = hm::twopass_cfg();
  hm::QueueCfg &qc = hm::queue_cfg();
  const hm::TwoPassCfg saved = cfg;
  const hm::QueueCfg qsaved = qc;
  const int pi = precision == HM_FP64 ? 0 : 1;
  const uint64_t per_x = (len / 2) * (precision == HM_FP64 ? sizeof(double2) : sizeof(float2));
  const uint64_t rows = len / 2 / 1024;  // pass-1 units per X-string
  // sample: at least 8 batches of the largest candidate and about 8192 pass-1 units
  uint64_t xmax = 1;
  while (xmax < 256 && 2 * (xmax * 2) * per_x <= (1ull << 30)) xmax *= 2;
  uint64_t sample = std::max<uint64_t>(8 * xmax, (8192 + rows - 1) / rows);
  if (1024 + sample > len) sample = len - 1024;
  hm::QReq q;
  q.nq = 1;
  q.q[0] = 2.0;
  double dd[10], best = 1e300;
  int bx = 0, beng = 1, bcps = 0;
  int rc = HM_OK;
  auto timeit = [&](double *t) {
    *t = 1e300;
    for (int rep = 0; rep < 2 && rc == HM_OK; ++rep) {
      rc = hm::run_sre(c, (const double2 *)c->d_psi, n, 1024, 1024 + sample, q, precision, dd);
      if (rc == HM_OK && rep > 0) *t = std::min(*t, c->last_ms);
    }
  };
  // stage kernels: every power of two up to xmax and the sizes 1.25 and 1.5 times one
  // (the kernel decodes its units with a division, so any X works; at n = 20 in FP64
  // X = 10 beats both 8 and 16)
  std::vector<uint64_t> xs;
  for (uint64_t P = 1; P <= xmax; P *= 2)
    for (uint64_t X : {P, P + P / 4, P + P / 2})
      if (X <= xmax && (xs.empty() || X > xs.back())) xs.push_back(X);
  qc.engine = 1;
  for (size_t xi = 0; xi < xs.size() && rc == HM_OK; ++xi) {
    const uint64_t X = xs[xi];
    cfg.X = (int)X;
    cfg.X_set = 1;
    cfg.ring_mib = std::max<int>(saved.ring_mib, (int)((2 * X * per_x + (1 << 20) - 1) >> 20));
    double t;
    timeit(&t);
    if (rc == HM_OK && t < best) {
      best = t;
      bx = (int)X;
      beng = 1;
      bcps = 0;
    }
  }
  cfg.X_set = saved.X_set;
  cfg.X = saved.X;
  cfg.ring_mib = saved.ring_mib;
  // queue sweep (4 slots of X X-strings each)
  qc.engine = 2;
  for (int cps = 0; cps <= 1 && rc == HM_OK; ++cps)
    for (uint64_t X = 1; 4 * X * per_x <= (1ull << 30) && X <= 256 && rc == HM_OK; X *= 2) {
      qc.X = (int)X;
      qc.X_set = 1;
      qc.ctas_per_sm = cps;
      double t;
      timeit(&t);
      if (rc == HM_OK && t < best) {
        best = t;
        bx = (int)X;
        beng = 2;
        bcps = cps;
      }
    }
  // restore the knobs; keep the results in the tables
  int tx[2][32], qx[2][32], qcps[2][32], qeng[2][32];
  memcpy(tx, cfg.tuned_x, sizeof tx);
  memcpy(qx, qc.tuned_x, sizeof qx);
  memcpy(qcps, qc.tuned_cps, sizeof qcps);
  memcpy(qeng, qc.tuned_engine, sizeof qeng);
  cfg = saved;
  qc = qsaved;
  memcpy(cfg.tuned_x, tx, sizeof tx);
  memcpy(qc.tuned_x, qx, sizeof qx);
  memcpy(qc.tuned_cps, qcps, sizeof qcps);
  memcpy(qc.tuned_engine, qeng, sizeof qeng);
  if (rc != HM_OK) return rc;
  qc.tuned_engine[pi][n] = beng;
  if (beng == 1) {
    cfg.tuned_x[pi][n] = bx;
  } else {
    qc.tuned_x[pi][n] = bx;
    qc.tuned_cps[pi][n] = bcps;
  }
  *best_x = bx;
  *best_us_per_x = best * 1e3 / (double)sample;
  return HM_OK;
}

extern "C" int hm_autotune_choice(int n, int precision, int *engine, int *batch, int *ctas_per_sm) {
  if (!engine || !batch || !ctas_per_sm) return HM_ERR_ARG;
  if (n < 0 || n >= 32 || (precision != HM_FP64 && precision != HM_FP32)) return HM_ERR_ARG;
  const int pi = precision == HM_FP64 ? 0 : 1;
  const hm::QueueCfg &qc = hm::queue_cfg();
  *engine = qc.tuned_engine[pi][n];
  *batch = *engine == 2 ? qc.tuned_x[pi][n] : (*engine == 1 ? hm::twopass_cfg().tuned_x[pi][n] : 0);
  *ctas_per_sm = *engine == 2 ? qc.tuned_cps[pi][n] : 0;
  return HM_OK;
}

extern "C" int hm_set_param(int param, int value) {
  hm::TwoPassCfg &cfg = hm::twopass_cfg();
  const hm::TwoPassCfg def;
  switch (param) {
    case HM_PARAM_BATCH:
      if (value == 0) {
        cfg.X_set = 0;
        hm::queue_cfg().X_set = 0;
        return HM_OK;
      }
      if (value < 1 || value > 4096) return HM_ERR_ARG;
      cfg.X = value;
      cfg.X_set = 1;
      hm::queue_cfg().X = value;
      hm::queue_cfg().X_set = 1;
      return HM_OK;
    case HM_PARAM_UNITS:
      if (value == 0) value = def.units_target;
      if (value < 256 || value > (1 << 20)) return HM_ERR_ARG;
      cfg.units_target = value;
      return HM_OK;
    case HM_PARAM_RING:
      if (value == 0) value = def.ring_mib;
      if (value < 8 || value > 4096) return HM_ERR_ARG;
      cfg.ring_mib = value;
      return HM_OK;
    case HM_PARAM_GRAPH:
      if (value == 0) value = def.graph_stages;
      if (value < 1 || value > 1024) return HM_ERR_ARG;
      cfg.graph_stages = value;
      return HM_OK;
    case HM_PARAM_ADJ_BATCH:
      if (value < 0 || value > 1024 || (value & (value - 1))) return HM_ERR_ARG;
      cfg.adj_x = value;
      return HM_OK;
    case HM_PARAM_ENGINE:
      if (value < 0 || value > 2) return HM_ERR_ARG;
      hm::queue_cfg().engine = value;
      return HM_OK;
    case HM_PARAM_QUEUE_SLOTS:
      if (value == 0) value = hm::QueueCfg().K;
      if (value < 2 || value > 64) return HM_ERR_ARG;
      hm::queue_cfg().K = value;
      return HM_OK;
    case HM_PARAM_QUEUE_SLOT_MIB:
      if (value == 0) value = hm::QueueCfg().slot_mib;
      if (value < 1 || value > 4096) return HM_ERR_ARG;
      hm::queue_cfg().slot_mib = value;
      return HM_OK;
    case HM_PARAM_QUEUE_CHUNK:
      if (value == 0) value = hm::QueueCfg().chunk;
      if (value < 1 || value > 64) return HM_ERR_ARG;
      hm::queue_cfg().chunk = value;
      return HM_OK;
    case HM_PARAM_QUEUE_CTAS:
      if (value < 0 || value > 32) return HM_ERR_ARG;
      hm::queue_cfg().ctas_per_sm = value;
      return HM_OK;
    case HM_PARAM_BATCH_SPLIT_N:
      if (value == 0) value = hm::QueueCfg().batch_split_n;
      if (value < 1 || value > 22) return HM_ERR_ARG;
      hm::queue_cfg().batch_split_n = value;
      return HM_OK;
    case HM_PARAM_QUEUE_LEAD:
      if (value == 0) value = hm::QueueCfg().lead;
      if (value < 1 || value > 16) return HM_ERR_ARG;
      hm::queue_cfg().lead = value;
      return HM_OK;
    case HM_PARAM_QUEUE_STALL_TEST:
      if (value < 0 || value > 1) return HM_ERR_ARG;
      hm::queue_cfg().stall_test = value;
      return HM_OK;
    default:
      return HM_ERR_ARG;
  }
}
