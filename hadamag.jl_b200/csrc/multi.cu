// multi.cu -- exact SRE over several GPUs in one call: one host thread and one context per
// listed device, each sweeping its contiguous share of the Gray range.
//
// Mirrors the per-rank part of ext/HadaMAGMPICUDAExt.jl:30-99: the rank's X-string range is
// split into nearly equal contiguous ranges (split_ranges, ext/HadaMAGMPICUDAExt.jl:8-28:
// the first N mod k parts one longer), one per GPU, each GPU runs its share with its own
// workspace from its own host thread (parts listed on the same device share its thread and
// run in list order), and the per-GPU sums are added.  Here each share is
// a hm_sre_range_dev call on that device's context and the shares' double-double sums are
// added in device-list order, so the result does not depend on which GPU finishes first.
// A caller with several processes (MPI ranks) passes its own rank's range to
// hm_sre_range_multi and reduces the returned double-double sums across ranks.
#include <math.h>

#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "hm_ctx.h"

namespace {

std::mutex g_multi_mu;                 // one multi-GPU call at a time
std::vector<hm_ctx *> g_multi_ctx;     // context per position of the device list
std::vector<int> g_multi_dev;          // device of each cached context
thread_local std::string g_multi_err;  // last error of this thread's multi-GPU call

int multi_fail(int code, const std::string &msg) {
  g_multi_err = msg;
  return code;
}

void dd_add(double *a, double bh, double bl) {
  const double s = a[0] + bh;
  const double bb = s - a[0];
  const double err = (a[0] - (s - bb)) + (bh - bb);
  const double lo = a[1] + bl + err;
  a[0] = s + lo;
  a[1] = lo - (a[0] - s);
}

}  // namespace

extern "C" {

int hm_sre_range_multi(const int *devices, int ndev, const double *psi, int n, uint64_t k_begin, uint64_t k_end,
                       const double *qs, int nq, int precision, double *p2_dd, double *m_dd) {
  g_multi_err.clear();
  if (!devices || ndev < 1 || ndev > 64) return multi_fail(HM_ERR_ARG, "need 1 <= ndev <= 64 devices");
  if (!psi || !qs || !p2_dd || !m_dd) return multi_fail(HM_ERR_ARG, "null pointer");
  if (n < 1 || n > 24) return multi_fail(HM_ERR_SIZE, "n outside [1, 24]");
  if (nq < 1 || nq > 4) return multi_fail(HM_ERR_ARG, "need 1 <= nq <= 4 Renyi indices");
  if (k_begin > k_end || k_end > (1ull << n)) return multi_fail(HM_ERR_ARG, "Gray range outside [0, 2^n)");
  std::lock_guard<std::mutex> lock(g_multi_mu);
  // split_ranges: k = min(ndev, N) parts, the first N mod k one longer
  const uint64_t N = k_end - k_begin;
  const int parts = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)ndev, N));
  const uint64_t base = N / parts, rem = N % parts;
  std::vector<uint64_t> kb(parts), ke(parts);
  uint64_t start = k_begin;
  for (int i = 0; i < parts; ++i) {
    kb[i] = start;
    ke[i] = start + base + ((uint64_t)i < rem ? 1 : 0);
    start = ke[i];
  }
  if ((int)g_multi_ctx.size() < parts) {
    g_multi_ctx.resize(parts, nullptr);
    g_multi_dev.resize(parts, -1);
  }
  for (int i = 0; i < parts; ++i) {
    if (g_multi_ctx[i] && g_multi_dev[i] != devices[i]) {
      hm_destroy(g_multi_ctx[i]);
      g_multi_ctx[i] = nullptr;
    }
    if (!g_multi_ctx[i]) {
      const int rc = hm_create(&g_multi_ctx[i], devices[i]);
      if (rc != HM_OK) return multi_fail(rc, "hm_create failed for device " + std::to_string(devices[i]));
      g_multi_dev[i] = devices[i];
    }
  }
  const int w = 2 * nq;
  std::vector<double> p2(2 * parts, 0.0), m((size_t)w * parts, 0.0);
  std::vector<int> rcs(parts, HM_OK);
  // one host thread per distinct device; parts that share a device run one after another
  // on that device's thread (kernels of one GPU gain nothing from running side by side)
  std::vector<int> owner(parts, -1);
  std::vector<std::vector<int>> groups;
  for (int i = 0; i < parts; ++i) {
    for (size_t g = 0; g < groups.size(); ++g)
      if (devices[groups[g][0]] == devices[i]) owner[i] = (int)g;
    if (owner[i] < 0) {
      owner[i] = (int)groups.size();
      groups.emplace_back();
    }
    groups[owner[i]].push_back(i);
  }
  std::vector<std::thread> th;
  for (size_t g = 0; g < groups.size(); ++g)
    th.emplace_back([&, g] {
      for (int i : groups[g])
        rcs[i] = hm_sre_range(g_multi_ctx[i], psi, n, kb[i], ke[i], qs, nq, precision, &p2[2 * i], &m[(size_t)w * i]);
    });
  for (auto &t : th) t.join();
  for (int i = 0; i < parts; ++i)
    if (rcs[i] != HM_OK)
      return multi_fail(rcs[i], "device " + std::to_string(devices[i]) + ": " + hm_last_error(g_multi_ctx[i]));
  p2_dd[0] = p2_dd[1] = 0.0;
  for (int j = 0; j < w; ++j) m_dd[j] = 0.0;
  for (int i = 0; i < parts; ++i) {
    dd_add(p2_dd, p2[2 * i], p2[2 * i + 1]);
    for (int t = 0; t < nq; ++t) dd_add(m_dd + 2 * t, m[(size_t)w * i + 2 * t], m[(size_t)w * i + 2 * t + 1]);
  }
  return HM_OK;
}

int hm_sre_multi(const int *devices, int ndev, const double *psi, int n, const double *qs, int nq, int precision,
                 double *out_sre, double *out_lost) {
  if (!out_sre || !out_lost) return multi_fail(HM_ERR_ARG, "null output pointer");
  if (n < 1 || n > 24) return multi_fail(HM_ERR_SIZE, "n outside [1, 24]");
  double p2[2], m[8];
  const int rc = hm_sre_range_multi(devices, ndev, psi, n, 0, 1ull << n, qs, nq, precision, p2, m);
  if (rc != HM_OK) return rc;
  const double dim = ldexp(1.0, n);
  for (int i = 0; i < nq; ++i) out_sre[i] = -log2((m[2 * i] + m[2 * i + 1]) / dim);
  *out_lost = fabs(1.0 - (p2[0] + p2[1]) / dim);
  return HM_OK;
}

const char *hm_multi_last_error(void) { return g_multi_err.c_str(); }

int hm_multi_release(void) {
  std::lock_guard<std::mutex> lock(g_multi_mu);
  for (hm_ctx *c : g_multi_ctx)
    if (c) hm_destroy(c);
  g_multi_ctx.clear();
  g_multi_dev.clear();
  return HM_OK;
}

}  // extern "C"
