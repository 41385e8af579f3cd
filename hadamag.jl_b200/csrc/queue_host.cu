// queue_host.cu -- host side of the persistent queue sweep: queue layout, ring and tensor
// maps, one captured graph per call (clears, state table, sweep, fold, read-back).
#include <math.h>

#include <algorithm>
#include <vector>

#include "queue_launch.cuh"
#include "sre_launch.cuh"

namespace hm {

template <typename T, int QS>
int launch_queue_kernel(hm_ctx *c, const QArgs &a, int ctas_per_sm, long long total_units, int *nwarps);
template <typename T, int QS>
int queue_warps(hm_ctx *c, int ctas_per_sm, long long total_units, int *nwarps);

__global__ void k_queue_fold(const double *__restrict__ slots, int nwarps, int nstates, int nsum, double *out) {
  // one block per state: thread t folds warps t, t + blockDim, ..., then a fixed-shape tree
  __shared__ dd sh[256][5];
  const int s = blockIdx.x, t = threadIdx.x;
  dd acc[5];
  for (int u = 0; u < 5; ++u) acc[u] = dd{0.0, 0.0};
  for (int w = t; w < nwarps; w += blockDim.x) {
    const double *sl = slots + ((size_t)w * nstates + s) * 2 * nsum;
    for (int u = 0; u < nsum; ++u) dd_add_dd(acc[u], dd{sl[2 * u], sl[2 * u + 1]});
  }
  for (int u = 0; u < 5; ++u) sh[t][u] = acc[u];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (t < o)
      for (int u = 0; u < nsum; ++u) dd_add_dd(sh[t][u], sh[t + o][u]);
    __syncthreads();
  }
  if (t == 0)
    for (int u = 0; u < nsum; ++u) {
      out[(size_t)s * 2 * nsum + 2 * u] = sh[0][u].hi;
      out[(size_t)s * 2 * nsum + 2 * u + 1] = sh[0][u].lo;
    }
}

QueueCfg &queue_cfg() {
  static QueueCfg cfg;
  return cfg;
}

namespace {

template <typename T>
int launch_kind(hm_ctx *c, int kind, const QArgs &a, int cps, long long total, int *nw) {
  switch (kind) {
    case QS_Q2:
      return launch_queue_kernel<T, QS_Q2>(c, a, cps, total, nw);
    case QS_Q23:
      return launch_queue_kernel<T, QS_Q23>(c, a, cps, total, nw);
    default:
      return launch_queue_kernel<T, QS_GEN>(c, a, cps, total, nw);
  }
}
template <typename T>
int warps_kind(hm_ctx *c, int kind, int cps, long long total, int *nw) {
  switch (kind) {
    case QS_Q2:
      return queue_warps<T, QS_Q2>(c, cps, total, nw);
    case QS_Q23:
      return queue_warps<T, QS_Q23>(c, cps, total, nw);
    default:
      return queue_warps<T, QS_GEN>(c, cps, total, nw);
  }
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace

int queue_choose_qs(const QReq &q, QParams &qp, int *idx);  // sre_host.cu (choose_qs)

// FP32 copies of the two-pass states (psi32 set in the state table); blockIdx.y = state
// y0 + blockIdx.y
static __global__ void k_queue_psi_to_f32(const QState *__restrict__ st, int y0) {
  const QState s = st[y0 + blockIdx.y];
  if (!s.psi32) return;
  float2 *out = const_cast<float2 *>(s.psi32);
  const uint64_t len = 1ull << s.n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 v = s.psi[i];
    out[i] = make_float2((float)v.x, (float)v.y);
  }
}

int run_queue(hm_ctx *c, const QueueItem *items, int nitems, const QReq &q, int precision, double *out_dd) {
  if (nitems <= 0) return HM_OK;
  const bool fp64 = precision != HM_FP32;
  const size_t vbytes = fp64 ? sizeof(double2) : sizeof(float2);
  QParams qp;
  int idx[4];
  const int kind = queue_choose_qs(q, qp, idx);
  const int NQ = kind == QS_Q2 ? 1 : (kind == QS_Q23 ? 2 : 4);
  const int nsum = 1 + NQ;
  const QueueCfg &cfg = queue_cfg();

  // cost order: two-pass states first, then the one-warp states, larger first
  std::vector<int> order(nitems);
  for (int i = 0; i < nitems; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const double cx = ldexp((double)(items[x].ke - items[x].kb), items[x].n);
    const double cy = ldexp((double)(items[y].ke - items[y].kb), items[y].n);
    const bool tx = items[x].n >= 12, ty = items[y].n >= 12;
    if (tx != ty) return tx;
    return cx > cy;
  });
  // ring slot: X-strings of the largest two-pass state per batch from the tuned table or
  // the default slot size
  int nmax = 0;
  for (int i = 0; i < nitems; ++i)
    if (items[i].n >= 12 && items[i].ke > items[i].kb) nmax = std::max(nmax, items[i].n);
  long long slot_elems = 0;
  if (nmax > 0) {
    int X = cfg.X_set ? cfg.X : cfg.tuned_x[fp64 ? 0 : 1][nmax];
    if (X <= 0) X = (int)std::max<long long>(1, ((long long)cfg.slot_mib << 20) / ((long long)vbytes << (nmax - 1)));
    while (X & (X - 1)) X &= X - 1;  // a power of two
    slot_elems = (long long)X << (nmax - 1);
  }
  const int K = std::max(cfg.K, cfg.lead + 1);
  const int cps = cfg.ctas_per_sm > 0 ? cfg.ctas_per_sm : (nmax > 0 ? cfg.tuned_cps[fp64 ? 0 : 1][nmax] : 0);
  // queue layout
  std::vector<QState> st(nitems);
  long long total = 0;
  int qnext = 0;
  for (int oi = 0; oi < nitems; ++oi) {
    const QueueItem &it = items[order[oi]];
    QState &s = st[oi];
    memset(&s, 0, sizeof s);
    s.psi = it.psi;
    s.k_begin = it.kb;
    s.k_end = it.ke;
    s.n = it.n;
    s.u0 = total;
    const uint64_t len = it.ke - it.kb;
    if (len == 0) {
      s.u1 = total;
      continue;
    }
    if (it.n <= 11) {
      s.X = 1 << (11 - it.n);
      total += (long long)((len + s.X - 1) / s.X);
    } else {
      // a power of two (the kernel decodes units with shifts): the slot's capacity, or the
      // next power of two above a shorter range (its extra X-strings are inactive units)
      const long long xcap = slot_elems >> (it.n - 1);
      long long x = 1;
      while (x < (long long)len && x < xcap) x <<= 1;
      s.X = (int)x;
      s.lgX = 63 - __builtin_clzll((unsigned long long)x);
      s.nbatch = (int)((len + s.X - 1) / s.X);
      s.q0 = qnext;
      qnext += s.nbatch;
      total += 2LL * s.nbatch * ((long long)s.X << (it.n - 11));
    }
    s.u1 = total;
  }
  // FP32: the two-pass states' FP32 copies, back to back
  size_t f32_elems = 0;
  if (!fp64)
    for (int oi = 0; oi < nitems; ++oi)
      if (st[oi].n >= 12 && st[oi].u1 > st[oi].u0) f32_elems += (size_t)1 << st[oi].n;
  if (f32_elems) {
    HM_TRY(ensure_dev(c, &c->d_psi32, &c->psi32_cap, f32_elems * sizeof(float2)));
    size_t off = 0;
    for (int oi = 0; oi < nitems; ++oi)
      if (st[oi].n >= 12 && st[oi].u1 > st[oi].u0) {
        st[oi].psi32 = (const float2 *)c->d_psi32 + off;
        off += (size_t)1 << st[oi].n;
      }
  }
  int nwarps = 0;
  HM_TRY(fp64 ? warps_kind<double>(c, kind, cps, total, &nwarps)
              : warps_kind<float>(c, kind, cps, total, &nwarps));
  // pass-2 units of every global batch: a pass-1 unit reusing slot q mod K waits for
  // batch q - K, which may belong to another state with another unit count
  std::vector<unsigned> bunits((size_t)std::max(qnext, 1), 0u);
  for (int oi = 0; oi < nitems; ++oi)
    if (st[oi].n >= 12)
      for (int b = 0; b < st[oi].nbatch; ++b) bunits[(size_t)st[oi].q0 + b] = (unsigned)st[oi].X << (st[oi].n - 11);
  // device scratch: [state table, batch unit counts][done1][done2][head, err][slots][fold out]
  const size_t st_bytes = sizeof(QState) * nitems;
  const size_t tab_bytes = st_bytes + sizeof(unsigned) * bunits.size();
  const size_t b_st = align_up(tab_bytes, 256);
  const size_t b_cnt = align_up(sizeof(unsigned) * (size_t)std::max(qnext, 1), 256);
  const size_t b_head = 256;
  const size_t b_slots = align_up(sizeof(double) * 2 * nsum * (size_t)nwarps * nitems, 256);
  const size_t b_out = align_up(sizeof(double) * 2 * nsum * (size_t)nitems, 256);
  const size_t total_bytes = b_st + 2 * b_cnt + b_head + b_slots + b_out;
  HM_TRY(ensure_dev(c, &c->d_queue, &c->queue_cap, total_bytes));
  char *base = (char *)c->d_queue;
  QState *d_st = (QState *)base;
  unsigned *d_done1 = (unsigned *)(base + b_st);
  unsigned *d_done2 = (unsigned *)(base + b_st + b_cnt);
  unsigned long long *d_head = (unsigned long long *)(base + b_st + 2 * b_cnt);
  int *d_err = (int *)(base + b_st + 2 * b_cnt + 64);
  double *d_slots = (double *)(base + b_st + 2 * b_cnt + b_head);
  double *d_out = (double *)(base + b_st + 2 * b_cnt + b_head + b_slots);
  // pinned host mirror: [state table, batch unit counts][fold out][err]
  const size_t h_bytes = b_st + b_out + 256;
  HM_TRY(ensure_host(c, &c->h_pin, &c->h_pin_cap, h_bytes));
  char *hb = (char *)c->h_pin;
  memcpy(hb, st.data(), st_bytes);
  memcpy(hb + st_bytes, bunits.data(), sizeof(unsigned) * bunits.size());
  double *h_out = (double *)(hb + b_st);
  int *h_err = (int *)(hb + b_st + b_out);

  QArgs a;
  memset(&a, 0, sizeof a);
  a.st = d_st;
  a.bunits = (const unsigned *)(base + st_bytes);
  a.done1 = d_done1;
  a.done2 = d_done2;
  a.next = d_head;
  a.err = d_err;
  a.slots = d_slots;
  a.total = total;
  a.qp = qp;
  a.nstates = nitems;
  a.K = K;
  a.chunk = cfg.chunk;
  a.slot_elems = slot_elems;
  a.stall_test = cfg.stall_test;
  a.lead = cfg.lead;
  a.poll_limit = cfg.stall_test ? 4096 : QWAIT_POLLS;
  if (nmax > 0) {
    HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, (size_t)K * slot_elems * vbytes));
    a.ring = c->d_inter;
    for (int n = 12; n <= nmax; ++n) {
      const int ti = n - 12;
      const int HI = n - 11, C = 1 << (10 - HI), NT = 1024 / C;
      a.xcap[ti] = (int)(slot_elems >> (n - 1));
      a.geom[ti] = ring_tma_geom(C, NT);
      // a tile row narrower than 16 bytes (FP32 at n = 21) has no tensor map: plain stores
      a.tma[ti] = encode_ring_tmap(&a.tmap[ti], a.ring, fp64 ? 8 : 4, C, 1 << HI, NT, K * a.xcap[ti],
                                   ((uint64_t)1 << (n - 1)) * vbytes, a.geom[ti])
                      ? 1
                      : 0;
      if (!a.tma[ti] && 2 * C * (fp64 ? 8 : 4) >= 16)
        return set_err(c, HM_ERR_CUDA, "queue sweep: tensor map of the n = %d ring could not be encoded", n);
    }
  }
  // clears, state table, sweep, fold, read-back: one stream sequence (a single launch of
  // the sweep gains nothing from graph capture, whose instantiation costs more host time
  // than the whole sweep of a small state)
  int nw_launched = 0;
  HM_CUDA(c, cudaMemsetAsync(d_done1, 0, 2 * b_cnt + b_head + b_slots, c->stream));
  HM_CUDA(c, cudaMemcpyAsync(d_st, hb, tab_bytes, cudaMemcpyHostToDevice, c->stream));
  if (f32_elems) {
    // every two-pass state's FP32 copy in one launch (a block row per state, 65535 rows
    // per launch)
    const unsigned gx = (unsigned)std::max(1, c->num_sms * 4 / std::max(1, nitems));
    for (int y0 = 0; y0 < nitems; y0 += 65535) {
      k_queue_psi_to_f32<<<dim3(gx, (unsigned)std::min(65535, nitems - y0)), 256, 0, c->stream>>>(d_st, y0);
      c->launches += 1;
      HM_CUDA(c, cudaGetLastError());
    }
  }
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  HM_TRY(fp64 ? launch_kind<double>(c, kind, a, cps, total, &nw_launched)
              : launch_kind<float>(c, kind, a, cps, total, &nw_launched));
  if (nw_launched != nwarps)
    return set_err(c, HM_ERR_CUDA, "queue sweep: launched %d warps, sized the slots for %d", nw_launched, nwarps);
  k_queue_fold<<<nitems, 256, 0, c->stream>>>(d_slots, nw_launched, nitems, nsum, d_out);
  HM_CUDA(c, cudaGetLastError());
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_CUDA(c, cudaMemcpyAsync(h_out, d_out, sizeof(double) * 2 * nsum * nitems, cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaMemcpyAsync(h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  c->launches += 2;
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  if (*h_err)
    return set_err(c, HM_ERR_TIMEOUT, "queue sweep: a batch counter wait gave up (the results are not valid)");
  for (int oi = 0; oi < nitems; ++oi) {
    double *o = out_dd + (size_t)order[oi] * 2 * (1 + q.nq);
    const double *h = h_out + (size_t)oi * 2 * nsum;
    o[0] = h[0];
    o[1] = h[1];
    for (int i = 0; i < q.nq; ++i) {
      o[2 + 2 * i] = h[2 * idx[i]];
      o[3 + 2 * i] = h[2 * idx[i] + 1];
    }
  }
  return HM_OK;
}

}  // namespace hm
