// mc.cu -- MC_SRE: Metropolis chains over X-strings (src/SRE.jl:110-192,
// src/Backends/Threads.jl:161-221, Simpson of src/Helpers.jl:223-236).
//
// All Nbeta chains advance together.  One step is: evaluate m(x) and p2(x) of every
// chain's proposal with the warp engine of the exact-SRE sweep (one warp per chain for
// n <= 11; a pass-1 and a pass-2 kernel over (chain, row / tile) units otherwise), then
// one update kernel applies the acceptance rule of src/SRE.jl:172-186 on the device and
// forms the next proposal from the injected stream.  Kernel arguments do not change
// between steps (the step counter lives in device memory), so a block of steps is
// captured once as a CUDA graph and replayed.
#include <math.h>

#include <utility>
#include <vector>

#include "hm_ctx.h"
#include "sre_kernels.cuh"

namespace hm {

namespace {

struct Chain {
  uint64_t cur, prop;  // current X-string, proposal under evaluation
  double prob, m2, p2; // currPROB, currM2, currP2
  double sM2, sM2sq, sP2;
  double beta;
  double m_prop, p2_prop;  // result of the last evaluation (n <= 11 path)
  long long n;
};

struct McArgs {
  const double2 *psi;
  const double2 *psi_sw[16];  // two-pass relabelled copies
  double2 *inter;             // nbeta x 2^(n-1)
  double *part;               // nbeta x U x 2 (p2, m) per pass-2 tile
  Chain *ch;
  const uint64_t *pd;  // nbeta x nsamples
  const double *rs;
  long long *step;  // device step counter
  unsigned *upd_done;  // blocks of k_mc_update that finished the current step
  QParams qp;
  int n, nbeta, nsamples, U;  // nbeta: chains of this run
  int chain0, nbeta_grid;     // first chain's index in the beta grid of nbeta_grid points
  double p2_0, m0;  // x = 0 sample
};

// q = 2 or generic through QS_GEN
template <int QS>
__device__ __forceinline__ double moment_scale(const QParams &qp) {
  return QS == QS_Q2 ? 16.0 : pow_q_dev(4.0, qp.q[0]);
}

// n <= 11: one warp evaluates one chain's proposal (pairing bit anywhere, no relabelling)
template <int NB, int QS>
__global__ void __launch_bounds__(128) k_mc_fused(McArgs a) {
  constexpr int R = 32, LOGR = 5;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  allow_next_grid();
  wait_prior_grid();  // the previous update has written the proposals
  const int c = blockIdx.x * 4 + warp;
  if (c >= a.nbeta) return;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  if (*a.step >= a.nsamples) return;
  const uint64_t x = a.ch[c].prop;
  if (x == 0) return;  // a zero proposal is never accepted; its moments are not used
  const int j = 63 - __clzll((long long)x);
  double2 v[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const uint32_t e = (uint32_t)(i * 32 + lane);
    double2 f = make_double2(0.0, 0.0);
    if (e < (1u << NB)) {
      const uint64_t r = insert0(e, j);
      f = conj_mul(__ldg(a.psi + r), __ldg(a.psi + (r ^ x)));
    }
    v[i] = f;
  }
  if constexpr (NB > 5) reg_wht<R, 0, NB - 5>(v);
  transpose_ab<R>(v, sm, lane);
  reg_wht<R, 0, (NB < 5 ? NB : 5)>(v);
  double s[5];
  QParams qp = a.qp;
  qp.nq = 1;
  lane_moments<R, QS>(v, s, qp, sm, lane);
  const double p2 = warp_sum(s[0]) * 4.0, m = warp_sum(s[1]) * moment_scale<QS>(a.qp);
  if (lane == 0) {
    a.ch[c].p2_prop = p2;
    a.ch[c].m_prop = m;
  }
  (void)LOGR;
}

// n >= 12, pass 1: warp units (chain, row)
template <int HI>
__global__ void __launch_bounds__(128) k_mc_p1(McArgs a) {
  constexpr int R = 32, PB = 10;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  allow_next_grid();
  wait_prior_grid();  // the previous update has written the proposals
  if (*a.step >= a.nsamples) return;
  const long long u = (long long)blockIdx.x * 4 + warp;
  if (u >= (long long)a.nbeta * a.U) return;
  const int c = (int)(u / a.U);
  const uint64_t row = (uint64_t)(u % a.U);
  const uint64_t x = a.ch[c].prop;
  if (x == 0) return;
  XInfo xx;
  xx.active = 1;
  xx.sw = -1;
  xx.xt = x;
  xx.jt = 63 - __clzll((long long)x);
  if (xx.jt < PB) {
    xx.sw = xx.jt;
    xx.xt = (x ^ (1ull << xx.jt)) | (1ull << (a.n - 1));
    xx.jt = a.n - 1;
  }
  const double2 *src = xx.sw < 0 ? a.psi : a.psi_sw[xx.sw];
  p1_unit<R, HI, false>(src, xx, row, a.inter + (size_t)c * ((size_t)1 << (a.n - 1)), sm, lane);
}

// n >= 12, pass 2: warp units (chain, tile) -> part[chain][tile]
template <int HI, int QS>
__global__ void __launch_bounds__(128) k_mc_p2(McArgs a) {
  constexpr int R = 32, PB = 10;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  allow_next_grid();
  wait_prior_grid();  // pass 1 of this step has stored the rows
  if (*a.step >= a.nsamples) return;
  const long long u = (long long)blockIdx.x * 4 + warp;
  if (u >= (long long)a.nbeta * a.U) return;
  const int c = (int)(u / a.U);
  const uint64_t tile = (uint64_t)(u % a.U);
  if (a.ch[c].prop == 0) return;
  double s[5];
  QParams qp = a.qp;
  qp.nq = 1;
  p2_unit<R, HI, QS>(a.inter + (size_t)c * ((size_t)1 << (a.n - 1)) + (tile << PB), sm, lane, s, qp);
  const double p2 = warp_sum(s[0]) * 4.0, m = warp_sum(s[1]) * moment_scale<QS>(a.qp);
  if (lane == 0) {
    a.part[2 * u] = p2;
    a.part[2 * u + 1] = m;
  }
}

// Metropolis update of every chain (src/SRE.jl:164-186) and next proposal.  One warp per
// chain, MC_UPD_WARPS chains per block, as many blocks as the chains need: for n >= 12
// the warp's lanes fold the chain's per-tile partials (lane l takes tiles l, l + 32, ...
// in double-double, then a fixed butterfly; the order never changes), and lane 0 updates
// the chain.  The last block to finish advances the device step counter (a ticket taken
// with an atomic after a fence, so every block has read the counter before it moves;
// nothing waits).
constexpr int MC_UPD_WARPS = 4;
__global__ void __launch_bounds__(MC_UPD_WARPS * 32) k_mc_update(McArgs a, int folded) {
  allow_next_grid();
  wait_prior_grid();  // this step's evaluation has finished
  const long long t = *a.step;
  const int c = blockIdx.x * MC_UPD_WARPS + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (t < a.nsamples && c < a.nbeta) {
    Chain ch = a.ch[c];
    const uint64_t prop = ch.prop;
    double m_prop = 0.0, p2_prop = 0.0;
    if (prop != 0) {
      if (folded) {
        dd sp{0.0, 0.0}, sm{0.0, 0.0};
        for (int i = lane; i < a.U; i += 32) {
          dd_add(sp, a.part[2 * ((size_t)c * a.U + i)]);
          dd_add(sm, a.part[2 * ((size_t)c * a.U + i) + 1]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          dd op, om;
          op.hi = __shfl_xor_sync(0xffffffffu, sp.hi, o);
          op.lo = __shfl_xor_sync(0xffffffffu, sp.lo, o);
          om.hi = __shfl_xor_sync(0xffffffffu, sm.hi, o);
          om.lo = __shfl_xor_sync(0xffffffffu, sm.lo, o);
          dd_add_dd(sp, op);
          dd_add_dd(sm, om);
        }
        p2_prop = sp.hi + sp.lo;
        m_prop = sm.hi + sm.lo;
      } else {
        p2_prop = ch.p2_prop;
        m_prop = ch.m_prop;
      }
    }
    if (lane == 0) {
      p2_prop /= (double)(1ull << a.n);
      const double pb = pow(m_prop, ch.beta);
      const double r = a.rs[(size_t)c * a.nsamples + t];
      if ((r < pb / ch.prob) && (prop != 0)) {
        ch.cur = prop;
        ch.prob = pb;
        ch.m2 = -log2(m_prop);
        ch.p2 = p2_prop;
      }
      ch.sM2 += ch.m2;
      ch.sM2sq += ch.m2 * ch.m2;
      ch.sP2 += ch.p2;
      ch.n += 1;
      if (t + 1 < a.nsamples) ch.prop = ch.cur ^ a.pd[(size_t)c * a.nsamples + t + 1];
      a.ch[c] = ch;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned ticket = atomicAdd(a.upd_done, 1u);
    if (ticket == gridDim.x - 1) {
      *a.upd_done = 0;
      if (t < a.nsamples) *a.step = t + 1;
    }
  }
}

// initial chain state: currPROB = 1e-120, currM2 = 0, currP2 = p2_0, first proposal
__global__ void k_mc_init(McArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < a.nbeta) {
    Chain ch;
    ch.cur = 0;
    ch.prop = a.pd[(size_t)c * a.nsamples];
    ch.prob = 1e-120;
    ch.m2 = 0.0;
    ch.p2 = a.p2_0;
    ch.sM2 = ch.sM2sq = ch.sP2 = 0.0;
    ch.beta = (double)(a.chain0 + c) / (double)(a.nbeta_grid - 1);
    ch.m_prop = ch.p2_prop = 0.0;
    ch.n = 0;
    a.ch[c] = ch;
  }
  if (c == 0) {
    *a.step = 0;
    *a.upd_done = 0;
  }
}

// per-chain means and the Simpson combination -> out[0] = m2, out[1 + 3c ..] = (M2, M2ADD, P2)
__global__ void k_mc_finish(McArgs a, double *out, uint64_t *final_mask) {
  if (threadIdx.x != 0) return;
  const int nb = a.nbeta;
  const double h = 1.0 / (double)(nb - 1);
  double odd = 0.0, even = 0.0, odda = 0.0, evena = 0.0;
  const double m2add = a.m0 / (double)(1ull << a.n);
  for (int i = 0; i < nb; ++i) {
    const Chain ch = a.ch[i];
    const double M2 = ch.sM2 / (double)ch.n;
    out[1 + 3 * i] = M2;
    out[2 + 3 * i] = m2add;
    out[3 + 3 * i] = ch.sP2 / (double)ch.n;
    final_mask[i] = ch.cur;
    if (i > 0 && i < nb - 1) {
      if (i % 2 == 1) {
        odd += M2;
        odda += m2add;
      } else {
        even += M2;
        evena += m2add;
      }
    }
  }
  if (a.chain0 != 0 || nb != a.nbeta_grid) {
    out[0] = 0.0;  // a range of the grid: the caller combines all chains
    return;
  }
  const double M2_0 = out[1], M2_e = out[1 + 3 * (nb - 1)];
  const double I_res = (h / 3.0) * (M2_0 + M2_e + 4.0 * odd + 2.0 * even);
  const double I_add = (h / 3.0) * (m2add + m2add + 4.0 * odda + 2.0 * evena);
  out[0] = -log2(pow(2.0, -I_res) + I_add);
}

// One launch of a step kernel.  The kernels of consecutive steps are chained by
// programmatic dependent launch (the next grid is set up while this one runs); every kernel
// waits for its predecessor at its start, before any access to global memory, so the
// order of their effects is the plain stream order.  The first launch of a captured block
// is not chained: it waits for everything before it.
template <typename... P, typename... A>
static cudaError_t mc_launch(hm_ctx *c, bool chained, void (*kern)(P...), int blocks, int threads, size_t smem,
                             A &&...args) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(blocks);
  lc.blockDim = dim3(threads);
  lc.dynamicSmemBytes = smem;
  lc.stream = c->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = chained ? 1 : 0;
  return cudaLaunchKernelEx(&lc, kern, std::forward<A>(args)...);
}

template <int QS>
int mc_enqueue_step(hm_ctx *c, McArgs &a, bool first) {
  const int n = a.n;
  const int upd_blocks = (a.nbeta + MC_UPD_WARPS - 1) / MC_UPD_WARPS;
  if (n <= 11) {
    const int nb = n - 1;
    const size_t smem = 4 * 32 * 32 * sizeof(double2);
    const int blocks = (a.nbeta + 3) / 4;
#define HM_MCF(NBv)                                                                             \
  case NBv:                                                                                     \
    HM_CUDA(c, cudaFuncSetAttribute(k_mc_fused<NBv, QS>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                    (int)smem));                                                \
    HM_CUDA(c, mc_launch(c, !first, k_mc_fused<NBv, QS>, blocks, 128, smem, a));                 \
    break;
    switch (nb) {
      HM_MCF(0)
      HM_MCF(1)
      HM_MCF(2)
      HM_MCF(3)
      HM_MCF(4)
      HM_MCF(5)
      HM_MCF(6)
      HM_MCF(7)
      HM_MCF(8)
      HM_MCF(9)
      HM_MCF(10)
      default:
        return set_err(c, HM_ERR_SIZE, "MC: n = %d", n);
    }
#undef HM_MCF
    HM_CUDA(c, mc_launch(c, true, k_mc_update, upd_blocks, MC_UPD_WARPS * 32, 0, a, 0));
  } else {
    const int hi = n - 11;
    const size_t smem = 4 * 32 * 32 * sizeof(double2);
    const long long units = (long long)a.nbeta * a.U;
    const int blocks = (int)((units + 3) / 4);
#define HM_MCP(HIv)                                                                                     \
  case HIv:                                                                                             \
    HM_CUDA(c, cudaFuncSetAttribute(k_mc_p1<HIv>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    HM_CUDA(c, cudaFuncSetAttribute(k_mc_p2<HIv, QS>, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                    (int)smem));                                                           \
    HM_CUDA(c, mc_launch(c, !first, k_mc_p1<HIv>, blocks, 128, smem, a));                               \
    HM_CUDA(c, mc_launch(c, true, k_mc_p2<HIv, QS>, blocks, 128, smem, a));                             \
    break;
    switch (hi) {
      HM_MCP(1)
      HM_MCP(2)
      HM_MCP(3)
      HM_MCP(4)
      HM_MCP(5)
      HM_MCP(6)
      HM_MCP(7)
      HM_MCP(8)
      HM_MCP(9)
      HM_MCP(10)
      default:
        return set_err(c, HM_ERR_SIZE, "MC: n = %d outside [1, 21]", n);
    }
#undef HM_MCP
    HM_CUDA(c, mc_launch(c, true, k_mc_update, upd_blocks, MC_UPD_WARPS * 32, 0, a, 1));
  }
  return HM_OK;
}

}  // namespace

int run_mc(hm_ctx *c, const double2 *psi, int n, double q, int nbeta_grid, int chain0, int nbeta, int nsamples,
           const uint64_t *pd_dev, const double *rs_dev, double p2_0, double m0, double *out /* 1 + 3 nbeta */,
           uint64_t *final_mask) {
  McArgs a;
  memset(&a, 0, sizeof a);
  a.psi = psi;
  a.n = n;
  a.nbeta = nbeta;
  a.chain0 = chain0;
  a.nbeta_grid = nbeta_grid;
  a.nsamples = nsamples;
  a.pd = pd_dev;
  a.rs = rs_dev;
  a.qp.q[0] = q;
  a.qp.nq = 1;
  const bool q2 = (q == 2.0);
  a.p2_0 = p2_0;
  a.m0 = m0;
  // device state: chains, step counter, per-tile partials, ring, relabelled copies
  const size_t len = (size_t)1 << n;
  if (n >= 12) {
    a.U = 1 << (n - 11);
    HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, (size_t)nbeta * (len / 2) * sizeof(double2)));
    a.inter = (double2 *)c->d_inter;
    HM_TRY(ensure_dev(c, &c->d_aux2, &c->aux2_cap, 10 * len * sizeof(double2)));
    k_psi_swapped<double2><<<c->num_sms * 8, 256, 0, c->stream>>>(psi, (double2 *)c->d_aux2, n, 10);
    c->launches += 1;
    for (int j = 0; j < 10; ++j) a.psi_sw[j] = (const double2 *)c->d_aux2 + (size_t)j * len;
  }
  const size_t part_bytes = (size_t)nbeta * (a.U > 0 ? a.U : 1) * 2 * sizeof(double);
  const size_t state_bytes = 256 + nbeta * sizeof(Chain) + part_bytes + (1 + 3 * nbeta) * sizeof(double) +
                             nbeta * sizeof(uint64_t) + 256;
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, state_bytes));
  char *base = (char *)c->d_out;
  a.step = (long long *)base;
  a.upd_done = (unsigned *)(base + 64);
  a.ch = (Chain *)(base + 256);
  a.part = (double *)(base + 256 + nbeta * sizeof(Chain));
  double *d_res = (double *)(base + 256 + nbeta * sizeof(Chain) + part_bytes);
  uint64_t *d_mask = (uint64_t *)(d_res + 1 + 3 * nbeta);
  k_mc_init<<<(nbeta + 127) / 128, 128, 0, c->stream>>>(a);
  c->launches += 1;
  HM_CUDA(c, cudaGetLastError());
  // capture a block of steps once, replay it
  const int G = 16;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  HM_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = HM_OK;
  for (int s = 0; s < G && rc == HM_OK; ++s)
    rc = q2 ? mc_enqueue_step<QS_Q2>(c, a, s == 0) : mc_enqueue_step<QS_GEN>(c, a, s == 0);
  cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
  if (rc != HM_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "MC graph capture failed: %s", cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "MC graph instantiation failed: %s", cudaGetErrorString(ce));
  for (int s = 0; s < nsamples; s += G) {
    ce = cudaGraphLaunch(exec, c->stream);
    if (ce != cudaSuccess) break;
    c->launches += G * (n <= 11 ? 2 : 3);  // per step: the sweep kernel(s) and the update
  }
  cudaGraphExecDestroy(exec);
  if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "MC graph launch failed: %s", cudaGetErrorString(ce));
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  k_mc_finish<<<1, 32, 0, c->stream>>>(a, d_res, d_mask);
  c->launches += 1;
  HM_CUDA(c, cudaGetLastError());
  HM_CUDA(c, cudaMemcpyAsync(out, d_res, (1 + 3 * nbeta) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (final_mask)
    HM_CUDA(c, cudaMemcpyAsync(final_mask, d_mask, nbeta * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  return HM_OK;
}

}  // namespace hm

namespace hm {
namespace {

// chains [cb, ce) of an nbeta-point grid; out: 1 + 3 (ce - cb) doubles
int mc_chains(hm_ctx *c, const double *psi, int n, double q, int nbeta, int cb, int ce, int nsamples,
              const uint64_t *prop_delta, const double *rs, double *out, uint64_t *final_mask) {
  if (!psi || !prop_delta || !rs) return set_err(c, HM_ERR_ARG, "null pointer");
  if (n < 1 || n > 21) return set_err(c, HM_ERR_SIZE, "MC: n = %d outside [1, 21]", n);
  if (nbeta < 3 || nbeta % 2 != 1 || nbeta > HM_MC_MAX_NBETA)
    return set_err(c, HM_ERR_ARG, "Simpson needs an odd number of beta points in [3, %d] (got %d)", HM_MC_MAX_NBETA,
                   nbeta);
  if (cb < 0 || ce > nbeta || cb >= ce)
    return set_err(c, HM_ERR_ARG, "chain range [%d, %d) outside the %d-point beta grid", cb, ce, nbeta);
  if (nsamples < 1) return set_err(c, HM_ERR_ARG, "nsamples must be >= 1");
  if (!(q >= 1.0 && q <= 16.0)) return set_err(c, HM_ERR_Q, "Renyi index q = %g outside [1, 16]", q);
  HM_CUDA(c, cudaSetDevice(c->device));
  c->launches = 0;
  const int nch = ce - cb;
  const size_t len = (size_t)1 << n;
  const size_t ns = (size_t)nch * nsamples;
  HM_TRY(ensure_dev(c, &c->d_psi, &c->psi_cap, len * sizeof(double2)));
  HM_CUDA(c, cudaMemcpyAsync(c->d_psi, psi, len * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  // m0 and p2_0 of x = 0 (sample_mask!(0), src/SRE.jl:147): one X-string of the exact
  // sweep, before the chains take the context's scratch buffers
  QReq qq;
  qq.nq = 1;
  qq.q[0] = q;
  double z[4];
  HM_TRY(run_sre(c, (const double2 *)c->d_psi, n, 0, 1, qq, HM_FP64, z));
  const double p2_0 = (z[0] + z[1]) / (double)len, m0 = z[2] + z[3];
  HM_TRY(ensure_dev(c, &c->d_aux, &c->aux_cap, ns * (sizeof(uint64_t) + sizeof(double))));
  uint64_t *pd = (uint64_t *)c->d_aux;
  double *r = (double *)(pd + ns);
  HM_CUDA(c, cudaMemcpyAsync(pd, prop_delta, ns * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
  HM_CUDA(c, cudaMemcpyAsync(r, rs, ns * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return run_mc(c, (const double2 *)c->d_psi, n, q, nbeta, cb, nch, nsamples, pd, r, p2_0, m0, out, final_mask);
}

}  // namespace
}  // namespace hm

extern "C" int hm_mc_sre(hm_ctx *c, const double *psi, int n, double q, int nbeta, int nsamples,
                         const uint64_t *prop_delta, const double *rs, double *out_m2, double *M2, double *M2ADD,
                         double *P2, uint64_t *final_mask) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!out_m2 || !M2 || !M2ADD || !P2) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  if (nbeta < 3 || nbeta > HM_MC_MAX_NBETA)
    return hm::set_err(c, HM_ERR_ARG, "Simpson needs an odd number of beta points in [3, %d] (got %d)",
                       HM_MC_MAX_NBETA, nbeta);
  std::vector<double> out(1 + 3 * (size_t)nbeta);
  HM_TRY(hm::mc_chains(c, psi, n, q, nbeta, 0, nbeta, nsamples, prop_delta, rs, out.data(), final_mask));
  *out_m2 = out[0];
  for (int i = 0; i < nbeta; ++i) {
    M2[i] = out[1 + 3 * i];
    M2ADD[i] = out[2 + 3 * i];
    P2[i] = out[3 + 3 * i];
  }
  return HM_OK;
}

extern "C" int hm_mc_sre_chains(hm_ctx *c, const double *psi, int n, double q, int nbeta, int chain_begin,
                                int chain_end, int nsamples, const uint64_t *prop_delta, const double *rs, double *M2,
                                double *M2ADD, double *P2, uint64_t *final_mask) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!M2 || !M2ADD || !P2) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  if (chain_begin < 0 || chain_end > nbeta || chain_begin >= chain_end || nbeta > HM_MC_MAX_NBETA)
    return hm::set_err(c, HM_ERR_ARG, "chain range [%d, %d) outside the %d-point beta grid", chain_begin, chain_end,
                       nbeta);
  std::vector<double> out(1 + 3 * (size_t)(chain_end - chain_begin));
  HM_TRY(hm::mc_chains(c, psi, n, q, nbeta, chain_begin, chain_end, nsamples, prop_delta, rs, out.data(),
                       final_mask));
  for (int i = 0; i < chain_end - chain_begin; ++i) {
    M2[i] = out[1 + 3 * i];
    M2ADD[i] = out[2 + 3 * i];
    P2[i] = out[3 + 3 * i];
  }
  return HM_OK;
}
