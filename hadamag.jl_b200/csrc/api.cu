// api.cu -- C ABI of libhadamag_b200.so: context lifetime, argument checks, host<->device
// staging and result finishing for the exact-SRE entry points and the Gray tables.
#include <math.h>
#include <stdarg.h>

#include <algorithm>
#include <vector>

#include "hm_common.cuh"
#include "hm_ctx.h"

using namespace hm;

namespace {

int check_qs(hm_ctx *c, const double *qs, int nq, QReq &q) {
  if (!qs || nq < 1 || nq > 4) return set_err(c, HM_ERR_ARG, "need 1 <= nq <= 4 Renyi indices (got %d)", nq);
  q.nq = nq;
  for (int i = 0; i < nq; ++i) {
    if (!(qs[i] >= 1.0 && qs[i] <= 16.0))
      return set_err(c, HM_ERR_Q, "Renyi index q = %g outside the supported range [1, 16]", qs[i]);
    q.q[i] = qs[i];
  }
  return HM_OK;
}

int check_prec(hm_ctx *c, int precision) {
  if (precision != HM_FP64 && precision != HM_FP32 && precision != HM_PLAIN)
    return set_err(c, HM_ERR_ARG, "unknown precision selector %d", precision);
  return HM_OK;
}

int stage_psi(hm_ctx *c, const double *psi_host, uint64_t len, const double2 **out) {
  HM_TRY(ensure_dev(c, &c->d_psi, &c->psi_cap, len * sizeof(double2)));
  HM_CUDA(c, cudaMemcpyAsync(c->d_psi, psi_host, len * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  *out = (const double2 *)c->d_psi;
  return HM_OK;
}

int check_dev_ptr(hm_ctx *c, const void *p) {
  if (!p) return set_err(c, HM_ERR_ARG, "null device pointer");
  if (((uintptr_t)p) & 15u) return set_err(c, HM_ERR_ALIGN, "device pointer %p is not 16-byte aligned", p);
  return HM_OK;
}

int sre_finish(const double *dd, int n, int nq, double *out_sre, double *out_lost) {
  const double dim = ldexp(1.0, n);
  const double p2 = dd[0] + dd[1];
  for (int i = 0; i < nq; ++i) {
    const double m = dd[2 + 2 * i] + dd[3 + 2 * i];
    out_sre[i] = -log2(m / dim);
  }
  if (out_lost) *out_lost = fabs(1.0 - p2 / dim);
  return HM_OK;
}

// codes of the global indices off .. off + N - 1 and the 1-based flips inside that slice
__global__ void k_gray_binary(uint64_t *codes, int64_t *flips, uint64_t N, uint64_t off = 0) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < N; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t g = gray_code(off + k);
    codes[k] = g;
    if (k + 1 < N) flips[k] = (int64_t)__ffsll((long long)(g ^ gray_code(off + k + 1)));
  }
}

// integer_to_gray (src/Basis.jl:123-133): base-q digits least significant first, folded
// from the most significant digit down with a running shift.
__device__ void q_gray(uint64_t val, int q, int n, int64_t *out) {
  int64_t shift = 0;
  uint64_t pw = 1;
  for (int i = 0; i < n - 1; ++i) pw *= (uint64_t)q;
  for (int i = n - 1; i >= 0; --i) {
    const int64_t d = (int64_t)((val / pw) % (uint64_t)q);
    const int64_t g = (d + shift) % q;
    out[i] = g;
    shift += q - g;
    if (i > 0) pw /= (uint64_t)q;
  }
}

__global__ void k_gray_general(int64_t *xtab, int64_t *flips, uint64_t N, int q, int n, uint64_t off = 0) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < N; k += (uint64_t)gridDim.x * blockDim.x) {
    int64_t a[40], b[40];
    q_gray(off + k, q, n, a);
    for (int i = 0; i < n; ++i) xtab[k * n + i] = a[i];
    if (k + 1 < N) {
      q_gray(off + k + 1, q, n, b);
      int64_t pos = 0;
      for (int i = 0; i < n; ++i)
        if (a[i] != b[i]) {
          pos = i + 1;
          break;
        }
      flips[k] = pos;
    }
  }
}

// eight independent DADD chains per thread; the result is only stored under a condition
// that never holds, which keeps the chains live
__global__ void k_probe_dadd(double *out, int iters, double s) {
  double a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = threadIdx.x + j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = a[j] + s;
  }
  double t = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) t += a[j];
  if (t == -1.0) out[0] = t;
}

// FP32 counterpart: 16 independent add chains per thread (the FP32 add latency is shorter
// and its rate twice the FP64 rate, so more chains keep the pipe full)
__global__ void k_probe_fadd(float *out, int iters, float s) {
  float a[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) a[j] = threadIdx.x + j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 16; ++j) a[j] = a[j] + s;
  }
  float t = 0.0f;
#pragma unroll
  for (int j = 0; j < 16; ++j) t += a[j];
  if (t == -1.0f) out[0] = t;
}

}  // namespace

extern "C" {

int hm_abi_version(void) { return HM_ABI_VERSION; }

int hm_create(hm_ctx **out, int device) {
  if (!out) return HM_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return HM_ERR_CUDA;
  }
  hm_ctx *c = new hm_ctx();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return HM_ERR_CUDA;
  }
  c->stream = c->own_stream;
  *out = c;
  return HM_OK;
}

int hm_destroy(hm_ctx *c) {
  if (!c) return HM_ERR_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  void *dev[] = {c->d_psi, c->d_psi32, c->d_inter, c->d_partials, c->d_ctrl, c->d_out, c->d_aux, c->d_aux2,
                 c->d_queue};
  for (void *p : dev)
    if (p) cudaFree(p);
  if (c->h_out) cudaFreeHost(c->h_out);
  if (c->h_pin) cudaFreeHost(c->h_pin);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return HM_OK;
}

const char *hm_last_error(hm_ctx *c) { return c ? c->err.c_str() : "null context"; }

int hm_set_stream(hm_ctx *c, void *stream) {
  if (!c) return HM_ERR_ARG;
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return HM_OK;
}

int hm_last_launch_count(hm_ctx *c, long long *count) {
  if (!c || !count) return HM_ERR_ARG;
  *count = c->launches;
  return HM_OK;
}

int hm_probe_fp64_peak(hm_ctx *c, double *ops_per_s) {
  if (!c || !ops_per_s) return HM_ERR_ARG;
  c->err.clear();
  HM_CUDA(c, cudaSetDevice(c->device));
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, sizeof(double) * 16));
  const int blocks = c->num_sms * 8, threads = 256, iters = 8192;
  k_probe_dadd<<<blocks, threads, 0, c->stream>>>(c->d_out, 64, 1.0);  // warm-up
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  k_probe_dadd<<<blocks, threads, 0, c->stream>>>(c->d_out, iters, 1.0);
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_CUDA(c, cudaGetLastError());
  HM_CUDA(c, cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  *ops_per_s = (double)blocks * threads * iters * 8.0 / (ms * 1e-3);
  return HM_OK;
}

int hm_probe_fp32_peak(hm_ctx *c, double *ops_per_s) {
  if (!c || !ops_per_s) return HM_ERR_ARG;
  c->err.clear();
  HM_CUDA(c, cudaSetDevice(c->device));
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, sizeof(double) * 16));
  const int blocks = c->num_sms * 8, threads = 256, iters = 8192;
  k_probe_fadd<<<blocks, threads, 0, c->stream>>>((float *)c->d_out, 64, 1.0f);  // warm-up
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  k_probe_fadd<<<blocks, threads, 0, c->stream>>>((float *)c->d_out, iters, 1.0f);
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_CUDA(c, cudaGetLastError());
  HM_CUDA(c, cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  *ops_per_s = (double)blocks * threads * iters * 16.0 / (ms * 1e-3);
  return HM_OK;
}

int hm_last_kernel_ms(hm_ctx *c, double *ms) {
  if (!c || !ms) return HM_ERR_ARG;
  *ms = c->last_ms;
  return HM_OK;
}

int hm_sre_range_dev(hm_ctx *c, const double *psi_dev, int n, uint64_t kb, uint64_t ke, const double *qs, int nq,
                     int precision, double *p2_dd, double *m_dd) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  c->launches = 0;
  if (!p2_dd || !m_dd) return set_err(c, HM_ERR_ARG, "null output pointer");
  if (n < 1 || n > 24) return set_err(c, HM_ERR_SIZE, "n = %d outside [1, 24]", n);
  const uint64_t dim = 1ull << n;
  if (kb > ke || ke > dim) return set_err(c, HM_ERR_ARG, "Gray range [%llu, %llu) outside [0, 2^%d)",
                                          (unsigned long long)kb, (unsigned long long)ke, n);
  QReq q;
  HM_TRY(check_qs(c, qs, nq, q));
  HM_TRY(check_prec(c, precision));
  HM_TRY(check_dev_ptr(c, psi_dev));
  HM_CUDA(c, cudaSetDevice(c->device));
  double dd[10];
  HM_TRY(run_sre(c, (const double2 *)psi_dev, n, kb, ke, q, precision, dd));
  p2_dd[0] = dd[0];
  p2_dd[1] = dd[1];
  for (int i = 0; i < nq; ++i) {
    m_dd[2 * i] = dd[2 + 2 * i];
    m_dd[2 * i + 1] = dd[3 + 2 * i];
  }
  return HM_OK;
}

int hm_sre_range(hm_ctx *c, const double *psi, int n, uint64_t kb, uint64_t ke, const double *qs, int nq,
                 int precision, double *p2_dd, double *m_dd) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!psi) return set_err(c, HM_ERR_ARG, "null state pointer");
  if (n < 1 || n > 24) return set_err(c, HM_ERR_SIZE, "n = %d outside [1, 24]", n);
  HM_CUDA(c, cudaSetDevice(c->device));
  const double2 *d;
  HM_TRY(stage_psi(c, psi, 1ull << n, &d));
  return hm_sre_range_dev(c, (const double *)d, n, kb, ke, qs, nq, precision, p2_dd, m_dd);
}

int hm_sre_dev(hm_ctx *c, const double *psi_dev, int n, const double *qs, int nq, int precision, double *out_sre,
               double *out_lost) {
  if (!c) return HM_ERR_ARG;
  if (!out_sre) return set_err(c, HM_ERR_ARG, "null output pointer");
  double p2[2], m[8];
  HM_TRY(hm_sre_range_dev(c, psi_dev, n, 0, (n >= 1 && n <= 24) ? (1ull << n) : 0, qs, nq, precision, p2, m));
  double dd[10];
  dd[0] = p2[0];
  dd[1] = p2[1];
  for (int i = 0; i < nq; ++i) {
    dd[2 + 2 * i] = m[2 * i];
    dd[3 + 2 * i] = m[2 * i + 1];
  }
  return sre_finish(dd, n, nq, out_sre, out_lost);
}

int hm_sre(hm_ctx *c, const double *psi, int n, const double *qs, int nq, int precision, double *out_sre,
           double *out_lost) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!psi) return set_err(c, HM_ERR_ARG, "null state pointer");
  if (n < 1 || n > 24) return set_err(c, HM_ERR_SIZE, "n = %d outside [1, 24]", n);
  HM_CUDA(c, cudaSetDevice(c->device));
  const double2 *d;
  HM_TRY(stage_psi(c, psi, 1ull << n, &d));
  return hm_sre_dev(c, (const double *)d, n, qs, nq, precision, out_sre, out_lost);
}

int hm_sre_batched(hm_ctx *c, int nstates, const double *const *psis, const int *ns, const double *qs, int nq,
                   int precision, double *out_sre, double *out_lost) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (nstates < 0 || (nstates > 0 && (!psis || !ns || !out_sre || !out_lost)))
    return set_err(c, HM_ERR_ARG, "null pointer or negative state count");
  QReq q;
  HM_TRY(check_qs(c, qs, nq, q));
  HM_TRY(check_prec(c, precision));
  size_t total = 0;
  for (int s = 0; s < nstates; ++s) {
    if (!psis[s]) return set_err(c, HM_ERR_ARG, "state %d: null pointer", s);
    if (ns[s] < 1 || ns[s] > 24) return set_err(c, HM_ERR_SIZE, "state %d: n = %d outside [1, 24]", s, ns[s]);
    total += (size_t)1 << ns[s];
  }
  HM_CUDA(c, cudaSetDevice(c->device));
  // every state goes to the device in one staging buffer, then the states run back to
  // back on the context's stream
  HM_TRY(ensure_dev(c, &c->d_psi, &c->psi_cap, total * sizeof(double2)));
  size_t off = 0;
  for (int s = 0; s < nstates; ++s) {
    const size_t len = (size_t)1 << ns[s];
    HM_CUDA(c, cudaMemcpyAsync((double2 *)c->d_psi + off, psis[s], len * sizeof(double2), cudaMemcpyHostToDevice,
                               c->stream));
    off += len;
  }
  // states below the split size go through one persistent queue launch (FP32: plus one
  // FP64 launch of every state's x = 0 transform); from the split size up a state's own
  // sweep dwarfs a call's fixed cost and the stage kernels are faster per X-string than
  // the queue (no dead-tile write-back), so those states, n > 21 and the plain selector
  // run one state per call
  c->launches = 0;
  const int split_n = hm::queue_cfg().batch_split_n;
  auto queued = [&](int n) { return precision != HM_PLAIN && n < split_n && n <= 21; };
  std::vector<QueueItem> items;
  std::vector<int> where;
  off = 0;
  for (int s = 0; s < nstates; ++s) {
    const size_t len = (size_t)1 << ns[s];
    if (queued(ns[s])) {
      items.push_back(QueueItem{(const double2 *)c->d_psi + off, ns[s], 0, (uint64_t)len});
      where.push_back(s);
    }
    off += len;
  }
  std::vector<double> dd((size_t)nstates * 2 * (1 + nq));
  double total_ms = 0.0;
  long long launches = 0;
  if (!items.empty()) {
    std::vector<double> qdd(items.size() * 2 * (1 + nq));
    HM_TRY(run_queue_sre(c, items.data(), (int)items.size(), q, precision, qdd.data()));
    total_ms += c->last_ms;
    launches += c->launches;
    for (size_t i = 0; i < items.size(); ++i)
      std::copy(qdd.begin() + i * 2 * (1 + nq), qdd.begin() + (i + 1) * 2 * (1 + nq),
                dd.begin() + (size_t)where[i] * 2 * (1 + nq));
  }
  off = 0;
  for (int s = 0; s < nstates; ++s) {
    const size_t len = (size_t)1 << ns[s];
    if (!queued(ns[s])) {
      c->launches = 0;
      HM_TRY(run_sre(c, (const double2 *)c->d_psi + off, ns[s], 0, len, q, precision, dd.data() + (size_t)s * 2 * (1 + nq)));
      total_ms += c->last_ms;
      launches += c->launches;
    }
    off += len;
  }
  for (int s = 0; s < nstates; ++s) sre_finish(dd.data() + (size_t)s * 2 * (1 + nq), ns[s], nq, out_sre + (size_t)s * nq, out_lost + s);
  c->last_ms = total_ms;
  c->launches = launches;
  return HM_OK;
}

int hm_gray_table(hm_ctx *c, int n, uint64_t *codes, int64_t *flips) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (n < 0 || n > 30) return set_err(c, HM_ERR_SIZE, "n = %d outside [0, 30]", n);
  if (!codes || (!flips && n > 0)) return set_err(c, HM_ERR_ARG, "null output pointer");
  HM_CUDA(c, cudaSetDevice(c->device));
  const uint64_t N = 1ull << n;
  HM_TRY(ensure_dev(c, &c->d_aux, &c->aux_cap, N * sizeof(uint64_t)));
  HM_TRY(ensure_dev(c, &c->d_aux2, &c->aux2_cap, N * sizeof(int64_t)));
  const unsigned blocks = (unsigned)std::min<uint64_t>((N + 255) / 256, (uint64_t)c->num_sms * 8);
  k_gray_binary<<<blocks, 256, 0, c->stream>>>((uint64_t *)c->d_aux, (int64_t *)c->d_aux2, N);
  HM_CUDA(c, cudaGetLastError());
  HM_CUDA(c, cudaMemcpyAsync(codes, c->d_aux, N * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
  if (N > 1)
    HM_CUDA(c, cudaMemcpyAsync(flips, c->d_aux2, (N - 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  return HM_OK;
}

int hm_gray_table_general(hm_ctx *c, int n, int q, int64_t *xtab, int64_t *flips) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (q < 2 || q > 16 || n < 0 || n > 40) return set_err(c, HM_ERR_SIZE, "need 2 <= q <= 16, 0 <= n <= 40");
  double Nd = pow((double)q, n);
  if (Nd > (double)(1 << 26)) return set_err(c, HM_ERR_SIZE, "q^n = %g exceeds 2^26", Nd);
  const uint64_t N = (uint64_t)llround(Nd);
  if ((!xtab && n > 0) || (!flips && N > 1)) return set_err(c, HM_ERR_ARG, "null output pointer");
  HM_CUDA(c, cudaSetDevice(c->device));
  HM_TRY(ensure_dev(c, &c->d_aux, &c->aux_cap, (N * (n > 0 ? n : 1)) * sizeof(int64_t)));
  HM_TRY(ensure_dev(c, &c->d_aux2, &c->aux2_cap, N * sizeof(int64_t)));
  const unsigned blocks = (unsigned)std::min<uint64_t>((N + 255) / 256, (uint64_t)c->num_sms * 8);
  k_gray_general<<<blocks, 256, 0, c->stream>>>((int64_t *)c->d_aux, (int64_t *)c->d_aux2, N, q, n);
  HM_CUDA(c, cudaGetLastError());
  if (n > 0)
    HM_CUDA(c, cudaMemcpyAsync(xtab, c->d_aux, N * n * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  if (N > 1)
    HM_CUDA(c, cudaMemcpyAsync(flips, c->d_aux2, (N - 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  return HM_OK;
}

int hm_gray_table_split(hm_ctx *c, int n, int q, int rank, int P, int64_t *codes, int64_t *flips,
                        int64_t *code_off, int64_t *code_cnt) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (P < 1 || rank < 0 || rank >= P) return set_err(c, HM_ERR_ARG, "need 0 <= rank < P (got rank %d, P %d)", rank, P);
  if (q < 2 || q > 16 || n < 0 || n > 40) return set_err(c, HM_ERR_SIZE, "need 2 <= q <= 16, 0 <= n <= 40");
  const double Nd = pow((double)q, n);
  if (Nd > (double)(1ull << 30)) return set_err(c, HM_ERR_SIZE, "q^n = %g exceeds 2^30", Nd);
  if (!code_off || !code_cnt) return set_err(c, HM_ERR_ARG, "null output pointer");
  const uint64_t N = (uint64_t)llround(Nd);
  // partition_counts (src/Helpers.jl:18-23): the first N mod P slices one longer
  const uint64_t base = N / (uint64_t)P, rem = N % (uint64_t)P;
  const uint64_t cnt = base + ((uint64_t)rank < rem ? 1 : 0);
  const uint64_t off = (uint64_t)rank * base + std::min<uint64_t>((uint64_t)rank, rem);
  *code_off = (int64_t)off;
  *code_cnt = (int64_t)cnt;
  if (cnt == 0) return HM_OK;
  const int width = q == 2 ? 1 : n;
  if ((!codes && width > 0) || (!flips && cnt > 1)) return set_err(c, HM_ERR_ARG, "null output pointer");
  HM_CUDA(c, cudaSetDevice(c->device));
  HM_TRY(ensure_dev(c, &c->d_aux, &c->aux_cap, cnt * (width > 0 ? width : 1) * sizeof(int64_t)));
  HM_TRY(ensure_dev(c, &c->d_aux2, &c->aux2_cap, cnt * sizeof(int64_t)));
  const unsigned blocks = (unsigned)std::min<uint64_t>((cnt + 255) / 256, (uint64_t)c->num_sms * 8);
  if (q == 2)
    k_gray_binary<<<blocks, 256, 0, c->stream>>>((uint64_t *)c->d_aux, (int64_t *)c->d_aux2, cnt, off);
  else
    k_gray_general<<<blocks, 256, 0, c->stream>>>((int64_t *)c->d_aux, (int64_t *)c->d_aux2, cnt, q, n, off);
  HM_CUDA(c, cudaGetLastError());
  if (width > 0)
    HM_CUDA(c, cudaMemcpyAsync(codes, c->d_aux, cnt * width * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  if (cnt > 1)
    HM_CUDA(c, cudaMemcpyAsync(flips, c->d_aux2, (cnt - 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  return HM_OK;
}

}  // extern "C"
