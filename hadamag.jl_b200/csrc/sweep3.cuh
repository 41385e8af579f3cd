// sweep3.cuh -- the exact-SRE sweep for 22 <= n <= 24: three passes per X-string.
//
// The half-transform of one X-string has n - 1 = 21 .. 23 index bits, one more to three
// more than the two-pass engine covers (10 bits of a 1024-point row + 10 bits of a
// 1024-element tile).  The intermediate of an X-string is kept as 2^K sub-vectors of 2^20
// elements (K = n - 21), sub-vector s holding the rows whose top K bits are s, each in the
// two-pass engine's n = 21 tile-major layout (tile = row position p, 1024 rows each):
//   inter_x[s 2^20 + p 2^10 + rho_low]   for row rho = s 2^10 + rho_low, position p.
//   pass 1: gather + build + transform one 1024-point row (as the two-pass engine);
//   pass 2: load one 1024-element tile (one position of 1024 rows of one sub-vector),
//           transform the 10 row bits, store it back in place;
//   pass 3: for 2^10 / 2^K offsets, the 2^K values at that offset of every sub-vector:
//           transform the K top bits in registers, then the moment sums.
// Pass 2 stores its registers in the transpose's order (element R l + i at position
// 32 i + l): every sub-vector's tiles get the same permutation, so pass 3 still pairs the
// same logical element across sub-vectors, and the sums do not depend on positions.
//
// Stage t runs pass 1 of batch t, pass 2 of batch t - 1 and pass 3 of batch t - 2, with
// batch b in ring slot b mod 3; the stages are chained as the two-pass stage kernels are
// (graph replay, programmatic dependent launch, griddepcontrol.wait before the first
// access that depends on the previous stage).  Slot reuse: pass 1 of batch t writes the
// slot that pass 3 of batch t - 3 read in stage t - 1; pass 2 of batch t - 1 rewrites the
// rows pass 1 stored in stage t - 1; pass 3 of batch t - 2 reads what pass 2 stored in
// stage t - 1.  Pass 3 drops the lines it has read from L2 (discard.global.L2): the next
// write to them is pass 1 of batch t + 1, in the next launch, after griddepcontrol.wait.
//
// x = 0 is built with the top-bit pairing h = (|a|^2 + |b|^2, |a|^2 - |b|^2) in pass 1 and
// summed with scale 1; the host runs it in FP64 only (an FP32 call splits it off).
#pragma once
#include "sre_kernels.cuh"

namespace hm {

struct Stage3Args {
  CUtensorMap tmap;  // tensor view of the ring as 3 X 2^K sub-vectors of the n = 21 layout
  const void *psi;
  const void *psi_sw[16];
  void *ring;
  double *slots;     // per warp: 2 (1 + NQ) doubles
  unsigned *stage;   // [0] stage index of node 0 of the current graph replay
  uint64_t k_begin, k_end;
  QParams qp;
  TmaGeom g;
  int n, X, nbatch, tma;
  int node;
};

// pass 2 of the three-pass sweep: transform one tile over its 10 row bits, in place
template <int R, typename V, typename Ready>
__device__ __forceinline__ void p2_store_unit(V *tile, V *sm, int lane, const Ready &ready) {
  constexpr int LOGR = ilog2c(R);
  V v[R];
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = __ldcg(tile + i * 32 + lane);
  reg_wht<R, 0, LOGR>(v);
  ready();
  transpose_ab<R>(v, sm, lane);
  reg_wht<R, 0, 5>(v);
#pragma unroll
  for (int i = 0; i < R; ++i) __stcg(tile + i * 32 + lane, v[i]);
}

// pass 3: offsets [unit M, unit M + M) of every sub-vector (M = 32 R / 2^K); register
// s J + j (J = R / 2^K) holds sub-vector s, offset unit M + 32 j + lane
template <int R, int K, int QS, typename V, typename Ready>
__device__ __forceinline__ void p3_unit(const V *x_base, uint64_t unit, V *sm, int lane, double *s,
                                        const QParams &qp, const Ready &ready) {
  constexpr int LOGR = ilog2c(R), J = R >> K, M = (32 * R) >> K;
  const uint64_t m0 = unit * M;
  V v[R];
#pragma unroll
  for (int sv = 0; sv < (1 << K); ++sv)
#pragma unroll
    for (int j = 0; j < J; ++j) v[sv * J + j] = __ldcg(x_base + ((uint64_t)sv << 20) + m0 + j * 32 + lane);
  reg_wht<R, LOGR - K, LOGR>(v);  // the sub-vector bits
  ready();
  lane_moments<R, QS>(v, s, qp, sm, lane);
}

// pass 1 of the three-pass sweep: row rho (n - 11 bits) of X-string k, stored into
// sub-vector rho >> 10 at row rho & 1023, through tensor stores (tma) or plain stores
template <int R, typename V, typename Pre, typename Ready>
__device__ __forceinline__ void p1_unit3(const V *__restrict__ psi, const V *__restrict__ src, uint64_t x, int n,
                                         uint64_t k, uint64_t k_end, uint64_t rho, V *sm, int lane, bool tma,
                                         const void *tmap, const TmaGeom &g, int vx0, V *inter_x, const Pre &pre,
                                         const Ready &ready) {
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5;
  V v[R];
  if (x == 0) {
    // top-bit pairing: a = psi(r), b = psi(r + 2^(n-1)) for the row's 1024 indices r
    const V *rowA = psi + (rho << PB);
    const V *rowB = rowA + (1ull << (n - 1));
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint32_t e = (uint32_t)(i * 32 + lane);
      v[i] = zero_pair(ld_psi(rowA + e), ld_psi(rowB + e));
    }
  } else {
    const XInfo xi = make_xinfo(k, k_end, n, PB);
    p1_build<R, false>(v, src, xi, rho, sm, lane);  // registers only
  }
  reg_wht<R, 0, LOGR>(v);
  ready();
  transpose_ab<R>(v, sm, lane);
  reg_wht<R, 0, 5>(v);
  const uint64_t sv = rho >> 10, rl = rho & 1023;
  if (tma) {
    // register i of lane l holds element k = R l + i, kept at position p = 32 i + l
#pragma unroll
    for (int i = 0; i < R; ++i) sm[i * 32 + lane] = v[i];
    fence_proxy_async_smem();
    __syncwarp();
    pre();
    if (lane == 0) {
      for (int b2 = 0; b2 < g.nb2; ++b2)
        for (int b0 = 0; b0 < g.nb0; ++b0)
          tma_store_4d(tmap, sm + (size_t)b2 * g.box2 * g.C + (size_t)b0 * (g.box0 / 2), b0 * g.box0, (int)rl,
                       b2 * g.box2, vx0 + (int)sv);
      bulk_commit();
    }
  } else {
    pre();
    V *sub = inter_x + (sv << 20);
#pragma unroll
    for (int i = 0; i < R; ++i) __stcg(sub + ((size_t)(i * 32 + lane) << 10) + rl, v[i]);
  }
}

template <typename T, int R, int K, int QS>
__global__ void __launch_bounds__(SRE_WARPS * 32, StageOcc<T>::value)
    k_sre_stage3(const __grid_constant__ Stage3Args a) {
  using V = typename VT<T>::V;
  static_assert(R == 32 && K >= 1 && K <= 3, "three-pass sweep: 1024-point rows and tiles, 1 to 3 top bits");
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5, NQ = QSet<QS>::NQ;
  extern __shared__ __align__(1024) unsigned char smem_stage3[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *sm = reinterpret_cast<V *>(smem_stage3) + warp * (32 * R);
  allow_next_grid();
  const long long t = (long long)*(volatile unsigned *)a.stage + a.node;
  if (t > a.nbatch + 1) return;  // padding stages of the last graph replay
  const int gwarp = blockIdx.x * SRE_WARPS + warp;
  const int nwarps = gridDim.x * SRE_WARPS;
  const V *psi = reinterpret_cast<const V *>(a.psi);
  V *ring = reinterpret_cast<V *>(a.ring);
  const int n = a.n;
  const uint64_t xlen = 1ull << (n - 1);
  const long long U = 1ll << (n - 11);  // units per X-string in every pass
  const long long per = (long long)a.X * U;
  const long long n1 = (t < a.nbatch) ? per : 0;                    // pass 1 of batch t
  const long long n2 = (t >= 1 && t - 1 < a.nbatch) ? per : 0;      // pass 2 of batch t - 1
  const long long n3 = (t >= 2) ? per : 0;                          // pass 3 of batch t - 2
  constexpr bool LANE_ACC = sizeof(T) == 8;
  dd acc[NQ + 1];
#pragma unroll
  for (int q = 0; q <= NQ; ++q) acc[q] = dd{0.0, 0.0};
  auto pre = [] { wait_prior_grid(); };
  // per warp: one pass-1 unit first (its loads and butterflies overlap the previous
  // stage's tail), then pass 2, pass 3, and the rest of pass 1
  const long long nfirst = n1 < nwarps ? n1 : nwarps;
  for (long long u = gwarp; u < n1 + n2 + n3; u += nwarps) {
    int pass;
    long long r;
    if (u < nfirst) {
      pass = 1, r = u;
    } else if (u < nfirst + n2) {
      pass = 2, r = u - nfirst;
    } else if (u < nfirst + n2 + n3) {
      pass = 3, r = u - nfirst - n2;
    } else {
      pass = 1, r = u - n2 - n3;
    }
    const long long b = t - (pass - 1);
    const int xs = (int)(r % a.X);
    const uint64_t sub = (uint64_t)(r / a.X);  // row (pass 1), tile (pass 2), offset block (pass 3)
    const uint64_t k = a.k_begin + (uint64_t)b * a.X + xs;
    if (k >= a.k_end) continue;
    const int slotx = (int)(b % 3) * a.X + xs;
    V *inter_x = ring + (size_t)slotx * xlen;
    // the previous unit's tensor stores must have read the shared buffer before this unit
    // writes it (waited for right before the unit's first shared-memory access)
    auto ready = [&] {
      if (a.tma) {
        if (lane == 0) bulk_wait_read_all();
        __syncwarp();
      }
    };
    if (pass == 1) {
      const uint64_t x = gray_code(k);
      int sw = -1;
      if (x != 0) {
        const int jt = 63 - __clzll((long long)x);
        if (jt < PB) sw = jt;
      }
      const V *src = sw < 0 ? psi : reinterpret_cast<const V *>(a.psi_sw[sw]);
      p1_unit3<R>(psi, src, x, n, k, a.k_end, sub, sm, lane, a.tma != 0, &a.tmap, a.g, slotx << K, inter_x, pre,
                  ready);
    } else if (pass == 2) {
      wait_prior_grid();
      p2_store_unit<R>(inter_x + (sub << PB), sm, lane, ready);
    } else {
      wait_prior_grid();
      double s[NQ + 1];
      p3_unit<R, K, QS>(inter_x, sub, sm, lane, s, a.qp, ready);
      // the lines are dead once read: the slot's next write is pass 1 of batch t + 1, in
      // the next launch, after its griddepcontrol.wait on this one
      {
        constexpr int M = (32 * R) >> K, LPS = (int)(M * sizeof(V) / 128);  // lines per sub-vector
        const char *xb = reinterpret_cast<const char *>(inter_x + sub * M);
#pragma unroll
        for (int ln = lane; ln < (LPS << K); ln += 32)
          asm volatile("discard.global.L2 [%0], 128;" ::"l"(xb + ((size_t)(ln / LPS) << 20) * sizeof(V) +
                                                             (size_t)(ln % LPS) * 128)
                       : "memory");
      }
      const bool xz = gray_code(k) == 0;
      s[0] = xz ? s[0] : 4.0 * s[0];
#pragma unroll
      for (int q = 0; q < NQ; ++q) s[1 + q] *= q_scale<QS>(q, xz, a.qp);
      if constexpr (LANE_ACC) {
#pragma unroll
        for (int q = 0; q <= NQ; ++q) dd_add(acc[q], s[q]);
      } else {
#pragma unroll
        for (int q = 0; q <= NQ; ++q) dd_add(acc[q], warp_sum(s[q]));
      }
    }
  }
  if (LANE_ACC && n3 > 0) {
    // fixed-order butterfly reduction of the lanes' accumulators
#pragma unroll
    for (int q = 0; q <= NQ; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        dd other;
        other.hi = __shfl_xor_sync(0xffffffffu, acc[q].hi, o);
        other.lo = __shfl_xor_sync(0xffffffffu, acc[q].lo, o);
        dd_add_dd(acc[q], other);
      }
    }
  }
  if (lane == 0 && n3 > 0) {
    wait_prior_grid();  // the previous stage updates the same slot
    double *sl = a.slots + (size_t)gwarp * 2 * (NQ + 1);
#pragma unroll
    for (int q = 0; q <= NQ; ++q) {
      dd v{sl[2 * q], sl[2 * q + 1]};
      dd_add_dd(v, acc[q]);
      sl[2 * q] = v.hi;
      sl[2 * q + 1] = v.lo;
    }
  }
  // the ring rows this warp stored are complete before the grid ends
  if (a.tma && lane == 0) bulk_wait_all();
}

}  // namespace hm
