// sre_launch.cuh -- host launchers for the exact-SRE kernels (instantiated per precision
// in sre_fp64.cu / sre_fp32.cu).
#pragma once
#include "hm_ctx.h"
#include "sre_kernels.cuh"
#include "sweep3.cuh"

namespace hm {

// Tunables of the two-pass stage kernels (set through hm_set_param): a batch holds about
// `units_target` warp units per pass (X = units_target / 2^HI X-strings, or X when set
// explicitly), the two-batch ring stays within `ring_mib`, and `graph_stages` stages are
// captured per CUDA graph.  Every stage costs a fixed few microseconds (launch, the first
// loads of all warps at once, the tail), which favours large batches, while a ring that
// outgrows the 126 MB L2 costs DRAM traffic.  Where they pull apart (n >= 18) the default
// batch comes from `measured_x`, timed on B200 (us per X-string, stage kernels chained
// by programmatic dependent launch, dead tiles discarded):
//   FP64  n = 18: X = 32 (0.95; X = 24 1.01)  n = 19: X = 16 (1.89; X = 12 1.91, X = 4 1.94)
//         n = 20: X = 10 (3.86; X = 8 4.05, X = 12 3.91, X = 16 4.18)  n = 21: X = 2 (10.6; X = 3 14.5)
//   FP32  n = 18: X = 64 (0.49)  n = 19: X = 32 (1.02; X = 16 1.09)
//         n = 20: X = 8 (2.72; X = 10 2.74, X = 12 3.06)  n = 21: X = 2 (10.4; X = 4 11.2)
// Any X works (the kernel decodes units with a division); larger rings than the L2 can
// still win while the stage count falls.  hm_autotune measures and records a batch for the
// machine at hand; setting HM_PARAM_BATCH, _UNITS or _RING switches to the generic rule.
inline int measured_x(bool fp64, int n) {
  static const int f64[4] = {32, 16, 10, 2}, f32[4] = {64, 32, 8, 2};
  return (n >= 18 && n <= 21) ? (fp64 ? f64 : f32)[n - 18] : 0;
}

struct TwoPassCfg {
  int X = 0;
  int X_set = 0;
  int units_target = 4096;
  int ring_mib = 64;
  int graph_stages = 128;  // stages per captured graph (128: 0.4 % faster than 32 at n = 20)
  int adj_x = 0;  // X-strings per batch of the adjoint stage kernels (0: the default rule)
  // batch sizes chosen by hm_autotune, per precision (0 FP64, 1 FP32) and qubit count;
  // 0 = not tuned.  Used when HM_PARAM_BATCH is not set.
  int tuned_x[2][32] = {};
};

TwoPassCfg &twopass_cfg();

// Tensor map of the two-pass ring for the pass-1 tensor stores (see p1_unit_tma):
// scalar_bytes 8 (FP64) or 4 (FP32), C positions per tile row, U = 2^HI rows, T tiles,
// two_x = 2X (slot, X-string) pairs, x_stride_bytes = 2^(n-1) complex.  Returns false
// (and leaves the plain stores in use) when the geometry does not meet the unit's rules
// or the driver does not provide the encoder.
bool encode_ring_tmap(CUtensorMap *m, void *ring, int scalar_bytes, int C, int U, int T, int two_x,
                      uint64_t x_stride_bytes, const TmaGeom &g);

inline TmaGeom ring_tma_geom(int C, int T) {
  TmaGeom g;
  g.C = C;
  g.box0 = 2 * C <= 256 ? 2 * C : 256;
  g.nb0 = 2 * C / g.box0;
  g.box2 = g.nb0 > 1 ? 1 : (T < 256 ? T : 256);
  g.nb2 = T / g.box2;
  return g;
}

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
  c->launches += 1;
  HM_CUDA(c, cudaGetLastError());
  *nwarps_out = nwarps;
  return HM_OK;
}

// Launch the nst chained stage kernels of a sweep (node s runs stage s).  Up to 32 stages
// go out as direct launches: capturing and instantiating a graph costs more host time
// than it saves there (an n = 12 call is a handful of stages).  Longer
// sweeps replay a captured graph of G stages, with a one-thread kernel advancing the stage
// base in device memory after every replay.
template <typename Kern, typename Args>
static int run_stage_chain(hm_ctx *c, Kern kern, Args &a, int nst, int blocks, size_t smem, int G,
                           const char *what) {
  auto launch = [&](int s) {
    a.node = s;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(blocks);
    lc.blockDim = dim3(SRE_WARPS * 32);
    lc.dynamicSmemBytes = smem;
    lc.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = s > 0 ? 1 : 0;  // the first stage waits for everything before it
    return cudaLaunchKernelEx(&lc, kern, a);
  };
  cudaError_t ce = cudaSuccess;
  G = std::min(G, nst);
  if (nst <= std::min(G, 32)) {
    for (int s = 0; s < nst && ce == cudaSuccess; ++s) ce = launch(s);
    c->launches += nst;
    if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "%s launch failed: %s", what, cudaGetErrorString(ce));
    return HM_OK;
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  HM_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  for (int s = 0; s < G && ce == cudaSuccess; ++s) ce = launch(s);
  if (ce == cudaSuccess) {
    k_stage_advance<<<1, 1, 0, c->stream>>>(a.stage, (unsigned)G);
    ce = cudaGetLastError();
  }
  const cudaError_t ce_end = cudaStreamEndCapture(c->stream, &graph);
  if (ce == cudaSuccess) ce = ce_end;
  if (ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return set_err(c, HM_ERR_CUDA, "%s graph capture failed: %s", what, cudaGetErrorString(ce));
  }
  ce = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "%s graph instantiation failed: %s", what, cudaGetErrorString(ce));
  for (int s = 0; s < nst && ce == cudaSuccess; s += G) {
    ce = cudaGraphLaunch(exec, c->stream);
    c->launches += G + 1;
  }
  cudaGraphExecDestroy(exec);
  if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "%s graph launch failed: %s", what, cudaGetErrorString(ce));
  return HM_OK;
}

// Stage-kernel two-pass sweep (see k_sre_stage): X-strings per batch sized so that a
// pass holds about `units_target` warp units, ring of two batches, stages replayed from
// a captured CUDA graph.
template <typename T, int R, int HI, int QS>
static int launch_stages(hm_ctx *c, const SreArgs &a0, int *nwarps_out) {
  using V = typename VT<T>::V;
  const TwoPassCfg cfg = twopass_cfg();
  constexpr int PB = ilog2c(R) + 5, NQ = QSet<QS>::NQ;
  StageArgs a;
  memset(&a, 0, sizeof a);
  a.psi = a0.psi;
  a.k_begin = a0.k_begin;
  a.k_end = a0.k_end;
  a.qp = a0.qp;
  a.n = a0.n;
  const uint64_t U = 1ull << HI;
  const uint64_t len = a.k_end - a.k_begin;
  const TwoPassCfg def;
  const bool generic = cfg.X_set || cfg.units_target != def.units_target || cfg.ring_mib != def.ring_mib;
  uint64_t X, ring_mib = (uint64_t)cfg.ring_mib;
  const int tuned = cfg.tuned_x[sizeof(T) == 8 ? 0 : 1][a.n];
  const int measured = generic ? 0 : measured_x(sizeof(T) == 8, a.n);
  if (cfg.X_set) {
    X = (uint64_t)cfg.X;
  } else if (tuned > 0 || measured > 0) {
    X = (uint64_t)(tuned > 0 ? tuned : measured);
    ring_mib = std::max<uint64_t>(ring_mib, (2 * X * ((uint64_t)1 << (a.n - 1)) * sizeof(V) + (1 << 20) - 1) >> 20);
  } else {
    X = std::max<uint64_t>(1, (uint64_t)cfg.units_target / U);
  }
  // ring bytes 2 X 2^(n-1) sizeof(V) within the budget
  const uint64_t per_x = ((uint64_t)1 << (a.n - 1)) * sizeof(V);
  while (X > 1 && 2 * X * per_x > (ring_mib << 20)) X >>= 1;
  if (X > len) X = len;
  a.X = (int)X;
  a.nbatch = (int)((len + X - 1) / X);
  const size_t ring_bytes = 2 * (size_t)X * per_x;
  HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, ring_bytes));
  a.ring = c->d_inter;
  {
    constexpr int C = 1 << (PB - HI), NT = (1 << PB) / C;
    a.g = ring_tma_geom(C, NT);
    a.tma = encode_ring_tmap(&a.tmap, a.ring, (int)sizeof(T), C, 1 << HI, NT, 2 * (int)X, per_x, a.g) ? 1 : 0;
  }
  if (a.k_begin < (1ull << PB) && a.k_end > 1) {  // some 0 < x < 2^PB in the range
    const size_t slen = (size_t)1 << a.n;
    HM_TRY(ensure_dev(c, &c->d_aux2, &c->aux2_cap, (size_t)PB * slen * sizeof(V)));
    k_psi_swapped<V><<<c->num_sms * 8, 256, 0, c->stream>>>(reinterpret_cast<const V *>(a.psi),
                                                            reinterpret_cast<V *>(c->d_aux2), a.n, PB);
    c->launches += 1;
    HM_CUDA(c, cudaGetLastError());
    for (int j = 0; j < PB; ++j) a.psi_sw[j] = reinterpret_cast<const V *>(c->d_aux2) + (size_t)j * slen;
  }
  const size_t smem = (size_t)SRE_WARPS * 32 * R * sizeof(V);
  auto kern = k_sre_stage<T, R, HI, QS>;
  HM_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, SRE_WARPS * 32, smem));
  if (occ < 1) occ = 1;
  long long units = 2 * (long long)X * (long long)U;
  int blocks = c->num_sms * occ;
  if ((long long)blocks * SRE_WARPS > units) blocks = (int)((units + SRE_WARPS - 1) / SRE_WARPS);
  const int nwarps = blocks * SRE_WARPS;
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap, sizeof(double) * 2 * (NQ + 1) * (size_t)nwarps));
  HM_CUDA(c, cudaMemsetAsync(c->d_partials, 0, sizeof(double) * 2 * (NQ + 1) * (size_t)nwarps, c->stream));
  a.slots = c->d_partials;
  HM_TRY(ensure_dev(c, (void **)&c->d_ctrl, &c->ctrl_cap, 4 * sizeof(unsigned)));
  HM_CUDA(c, cudaMemsetAsync(c->d_ctrl, 0, 4 * sizeof(unsigned), c->stream));
  a.stage = c->d_ctrl;
  const int nst = a.nbatch + 1;
  HM_TRY(run_stage_chain(c, kern, a, nst, blocks, smem, cfg.graph_stages, "stage"));
  *nwarps_out = nwarps;
  return HM_OK;
}

// Three-pass sweep for n = 21 + K (K = 1 .. 3): batch X (HM_PARAM_BATCH, else about 4096
// units per pass: X = 2 at n = 22, 1 above), ring of three batches, graph replay of
// programmatically chained stages as launch_stages.
template <typename T, int R, int K, int QS>
static int launch_stages3(hm_ctx *c, const SreArgs &a0, int *nwarps_out) {
  using V = typename VT<T>::V;
  const TwoPassCfg cfg = twopass_cfg();
  constexpr int PB = ilog2c(R) + 5, NQ = QSet<QS>::NQ;
  Stage3Args a;
  memset(&a, 0, sizeof a);
  a.psi = a0.psi;
  a.k_begin = a0.k_begin;
  a.k_end = a0.k_end;
  a.qp = a0.qp;
  a.n = a0.n;
  const uint64_t U = 1ull << (a.n - 11);
  const uint64_t len = a.k_end - a.k_begin;
  uint64_t X = cfg.X_set ? (uint64_t)cfg.X : std::max<uint64_t>(1, 4096 / U);
  if (X > len) X = len;
  a.X = (int)X;
  a.nbatch = (int)((len + X - 1) / X);
  const uint64_t per_x = ((uint64_t)1 << (a.n - 1)) * sizeof(V);
  HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, 3 * (size_t)X * per_x));
  a.ring = c->d_inter;
  {
    // the ring as 3 X 2^K sub-vectors in the n = 21 layout: rows of C = 1 position,
    // 1024 rows, 1024 tiles
    a.g = ring_tma_geom(1, 1 << PB);
    a.tma = encode_ring_tmap(&a.tmap, a.ring, (int)sizeof(T), 1, 1 << PB, 1 << PB, (int)(3 * X) << K,
                             ((uint64_t)1 << 20) * sizeof(V), a.g)
                ? 1
                : 0;
  }
  if (a.k_begin < (1ull << PB) && a.k_end > 1) {  // some 0 < x < 2^PB in the range
    const size_t slen = (size_t)1 << a.n;
    HM_TRY(ensure_dev(c, &c->d_aux2, &c->aux2_cap, (size_t)PB * slen * sizeof(V)));
    k_psi_swapped<V><<<c->num_sms * 8, 256, 0, c->stream>>>(reinterpret_cast<const V *>(a.psi),
                                                            reinterpret_cast<V *>(c->d_aux2), a.n, PB);
    c->launches += 1;
    HM_CUDA(c, cudaGetLastError());
    for (int j = 0; j < PB; ++j) a.psi_sw[j] = reinterpret_cast<const V *>(c->d_aux2) + (size_t)j * slen;
  }
  const size_t smem = (size_t)SRE_WARPS * 32 * R * sizeof(V);
  auto kern = k_sre_stage3<T, R, K, QS>;
  HM_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, SRE_WARPS * 32, smem));
  if (occ < 1) occ = 1;
  const long long units = (long long)X * (long long)U;
  int blocks = c->num_sms * occ;
  if ((long long)blocks * SRE_WARPS > units) blocks = (int)((units + SRE_WARPS - 1) / SRE_WARPS);
  const int nwarps = blocks * SRE_WARPS;
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap, sizeof(double) * 2 * (NQ + 1) * (size_t)nwarps));
  HM_CUDA(c, cudaMemsetAsync(c->d_partials, 0, sizeof(double) * 2 * (NQ + 1) * (size_t)nwarps, c->stream));
  a.slots = c->d_partials;
  HM_TRY(ensure_dev(c, (void **)&c->d_ctrl, &c->ctrl_cap, 4 * sizeof(unsigned)));
  HM_CUDA(c, cudaMemsetAsync(c->d_ctrl, 0, 4 * sizeof(unsigned), c->stream));
  a.stage = c->d_ctrl;
  const int nst = a.nbatch + 2;
  HM_TRY(run_stage_chain(c, kern, a, nst, blocks, smem, cfg.graph_stages, "three-pass"));
  *nwarps_out = nwarps;
  return HM_OK;
}

#define HM_FUSED_CASE(NBv)                                         \
  case NBv:                                                        \
    return launch_fused<T, R, ((NBv) <= PB ? (NBv) : PB), QS>(c, a, nw);
#define HM_2P_CASE(HIv)                                            \
  case HIv:                                                        \
    return launch_stages<T, R, ((HIv) <= PB ? (HIv) : PB), QS>(c, a, nw);

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
      case 11:
        if constexpr (R == 32) return launch_stages3<T, R, 1, QS>(c, a, nw);
        break;
      case 12:
        if constexpr (R == 32) return launch_stages3<T, R, 2, QS>(c, a, nw);
        break;
      case 13:
        if constexpr (R == 32) return launch_stages3<T, R, 3, QS>(c, a, nw);
        break;
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
  return dispatch_sre<T, R, QS>(c, a, nwarps);
}

}  // namespace hm
