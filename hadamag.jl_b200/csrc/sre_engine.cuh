// sre_engine.cuh -- warp-level Walsh-Hadamard engine for the exact-SRE sweep.
//
// Mathematics (restating src/SRE.jl:424-540 and src/Helpers.jl:90 in a form that maps to
// registers).  For an X-string x the reference builds g_x(r) = Re f + Im f with
// f(r) = conj psi(r) psi(r ^ x), applies the unnormalised WHT over all n bits and sums
// F^2 and (F^2)^q.  Because f(r ^ x) = conj f(r), the n-bit transform of g splits into
// two (n-1)-bit transforms: pick a pairing bit j with x_j = 1, restrict r to the half
// V0 = {r : r_j = 0} and compress bit j away; then
//     { F(k) : k }  =  { 2 Re W(k'), 2 Im W(k') : k' }  with  W = WHT_{n-1}(f|V0)
// (Re W holds the k with even k.x, Im W the odd ones).  So one complex transform of
// 2^(n-1) points yields all 2^n values of F, with one butterfly stage and half of the
// gathers saved.  For x = 0 the pairing bit is the top bit and
//     h(r') = (|psi(r')|^2 + |psi(r'+2^(n-1))|^2,  |psi(r')|^2 - |psi(r'+2^(n-1))|^2)
// gives F = Re, Im of WHT_{n-1}(h) directly.
//
// Any GF(2)-linear relabelling of r permutes the outputs k; the sums over k do not see
// the permutation.  The two-pass kernels use this to move the pairing bit of x < 2^PB
// into the high part of the index (swap bit j with bit n-1).
//
// Data layout of one warp's tile (R complex per lane, 32R complex per warp):
//   layout A: lane l, register i  <->  element e = 32 i + l   (coalesced gathers)
//   layout B: lane l, register i  <->  element e = R l + i
// A transform over the bits held in registers needs no data movement; switching
// between A and B goes through a warp-private, XOR-swizzled shared-memory buffer
// (conflict-free 16-byte / 8-byte accesses).
#pragma once
#include "hm_common.cuh"
#ifdef HM_TMEM_EXCHANGE
#include "tmem_transpose.cuh"
#endif

namespace hm {

// ---------------------------------------------------------------------------------
// in-register butterflies over register-index bits [LO, HI)
template <int R, int LO, int HI, typename V>
__device__ __forceinline__ void reg_wht(V (&v)[R]) {
#pragma unroll
  for (int s = LO; s < HI; ++s) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      if ((i >> s) & 1) continue;
      const int k = i | (1 << s);
      const V a = v[i], b = v[k];
      v[i] = v_add(a, b);
      v[k] = v_sub(a, b);
    }
  }
}

// layout A -> layout B through a warp-private buffer of 32R elements
template <int R, typename V>
__device__ __forceinline__ void transpose_ab(V (&v)[R], V *sm, int lane) {
  constexpr int LOGR = ilog2c(R);
  constexpr int SW = 128 / (int)sizeof(V) - 1;  // slots per 128-byte bank row - 1
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int e = i * 32 + lane;
    sm[e ^ ((e >> LOGR) & SW)] = v[i];
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int e = lane * R + i;
    v[i] = sm[e ^ ((e >> LOGR) & SW)];
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------------
// Lane <-> register exchanges through tensor memory (tmem_transpose.cuh), compiled only
// with -DHM_TMEM_EXCHANGE.  A two-pass unit must move the five element bits held by the
// lane number into registers once per pass.  Through shared memory that is a 32 KB store +
// load per warp unit on the L1/shared data path, which the ring gathers and stores also
// use; through TMEM it is three (pass 1) or one to three (pass 2) store/load rounds on the
// tensor-memory path (about 3x the shared-memory rate on B200, and a separate datapath).
// Measured on B200 the exchanges give bit-identical results but make the sweep 1.5-1.7x
// slower: every round is a store, a wait, a load and a wait in series, about 700 cycles
// per warp, and 8 warps per SM cannot hide three of them per unit.  The product path
// therefore keeps the shared-memory transposes.  A CTA allocates the columns once; each
// warp uses its own 32 lanes (warp w of the CTA reaches lanes 32 (w mod 4) ..).
#ifdef HM_TMEM_EXCHANGE
template <typename T> struct TmemCols { static constexpr int value = sizeof(T) == 8 ? 128 : 64; };

__device__ __forceinline__ uint32_t tmem_cta_alloc(uint32_t *slot, int ncols) {
  if (threadIdx.x < 32) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return *(volatile uint32_t *)slot;
}

// every warp of the CTA must have finished its TMEM accesses
__device__ __forceinline__ void tmem_cta_free(uint32_t base, int ncols) {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (threadIdx.x < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// this warp's lanes of the CTA's allocation
__device__ __forceinline__ uint32_t tmem_warp_addr(uint32_t base) {
  return base + ((uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16);
}

// pass-1 row: lanes e0..e4 / registers e5..e9 in, registers e0..e4 out (register i =
// element bits of i), the lane number a fixed relabelling of e5..e9
__device__ __forceinline__ void tmem_row(double2 (&v)[32], uint32_t ta) { tmem_xchg_row_f64(v, ta); }
__device__ __forceinline__ void tmem_row(float2 (&v)[32], uint32_t ta) { tmem_xchg_row_f32(v, ta); }

// pass-2 tile of 2^HI rows (6 <= HI <= 10): the row bits on lanes go to registers, lowest
// row bit at register bit 0; afterwards register bits 0 .. HI - 6 hold the rows still to
// transform
template <int HI, typename V>
__device__ __forceinline__ void tmem_tile(V (&v)[32], uint32_t ta) {
  constexpr bool F64 = sizeof(V) == 16;
  if constexpr (HI == 6) {
    if constexpr (F64) tmem_xchg_tile6_f64(v, ta); else tmem_xchg_tile6_f32(v, ta);
  } else if constexpr (HI == 7) {
    if constexpr (F64) tmem_xchg_tile7_f64(v, ta); else tmem_xchg_tile7_f32(v, ta);
  } else if constexpr (HI == 8) {
    if constexpr (F64) tmem_xchg_tile8_f64(v, ta); else tmem_xchg_tile8_f32(v, ta);
  } else if constexpr (HI == 9) {
    if constexpr (F64) tmem_xchg_tile9_f64(v, ta); else tmem_xchg_tile9_f32(v, ta);
  } else if constexpr (HI == 10) {
    if constexpr (F64) tmem_xchg_tile10_f64(v, ta); else tmem_xchg_tile10_f32(v, ta);
  }
}
#endif  // HM_TMEM_EXCHANGE

// ---------------------------------------------------------------------------------
// element builders
template <typename V>
__device__ __forceinline__ V conj_mul(V a, V b) {  // conj(a) * b
  V r;
  r.x = fma(a.x, b.x, a.y * b.y);
  r.y = fma(a.x, b.y, -(a.y * b.x));
  return r;
}
template <typename V>
__device__ __forceinline__ V zero_pair(V a, V b) {  // x = 0: (|a|^2 + |b|^2, |a|^2 - |b|^2)
  const auto na = fma(a.x, a.x, a.y * a.y);
  const auto nb = fma(b.x, b.x, b.y * b.y);
  V r;
  r.x = na + nb;
  r.y = na - nb;
  return r;
}

template <typename V> __device__ __forceinline__ V ld_psi(const V *p) { return __ldg(p); }

// ---------------------------------------------------------------------------------
// moment sets: which sums a kernel accumulates besides sum F^2
enum { QS_Q2 = 1, QS_Q23 = 3, QS_GEN = 0 };
template <int QS> struct QSet {
  static constexpr int NQ = (QS == QS_Q2) ? 1 : (QS == QS_Q23 ? 2 : 4);
};

struct QParams {
  double q[4];
  int nq;
};

__device__ __forceinline__ double pow_q_dev(double y, double q) {
  // integer q in [1,16]: repeated squaring; otherwise pow
  if (q == floor(q) && q >= 1.0 && q <= 16.0) {
    int e = (int)q;
    double r = 1.0, b = y;
    while (e) {
      if (e & 1) r *= b;
      b *= b;
      e >>= 1;
    }
    return r;
  }
  return pow(y, q);
}

// Per-lane sums of F^2 and of (F^2)^q over the R complex registers (2R values of F/2
// for x != 0; the caller applies the 4 / 4^q scale), plain FP64 sums in a fixed order.
// Generic Renyi indices: the F values go through the warp's shared buffer so that the
// pow() evaluations run in a rolled loop instead of an unrolled register sweep.
template <int R, typename V>
__device__ __noinline__ void lane_moments_gen(const V *sm, int lane, double *s, const QParams &qp) {
  double a2 = 0.0, ag[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int i = 0; i < R; ++i) {
    const V f2 = sm[lane + 32 * i];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double f = c ? (double)f2.y : (double)f2.x;
      const double y = f * f;
      a2 += y;
#pragma unroll 1
      for (int t = 0; t < qp.nq; ++t) ag[t] += pow_q_dev(y, qp.q[t]);
    }
  }
  s[0] = a2;
#pragma unroll
  for (int t = 0; t < 4; ++t) s[1 + t] = ag[t];
}

// Both precisions take the powers and the sums in FP64: an FP32 value of F converts to
// double exactly, so the FP32 path's only roundings are those of f and of the butterflies.
// NA interleaved accumulators per sum (value j goes to accumulator j mod NA, combined
// pairwise at the end) keep the dependent-add chains short; the order is fixed.
template <int R, int QS, typename V>
__device__ __forceinline__ void lane_moments(const V (&v)[R], double *s, const QParams &qp, V *sm, int lane) {
  if constexpr (QS == QS_GEN) {
#pragma unroll
    for (int i = 0; i < R; ++i) sm[lane + 32 * i] = v[i];
    lane_moments_gen<R>(sm, lane, s, qp);
    __syncwarp();
    return;
  } else {
    constexpr int NA = 4;
    double a2[NA], a4[NA], a6[NA];
#pragma unroll
    for (int t = 0; t < NA; ++t) a2[t] = a4[t] = a6[t] = 0.0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const double f = c ? (double)v[i].y : (double)v[i].x;
        const double y = f * f;
        const int t = (2 * i + c) % NA;
        a2[t] += y;
        a4[t] = fma(y, y, a4[t]);
        if constexpr (QS == QS_Q23) a6[t] = fma(y * y, y, a6[t]);
      }
    }
#pragma unroll
    for (int w = NA / 2; w > 0; w >>= 1)
#pragma unroll
      for (int t = 0; t < w; ++t) {
        a2[t] += a2[t + w];
        a4[t] += a4[t + w];
        a6[t] += a6[t + w];
      }
    s[0] = a2[0];
    s[1] = a4[0];
    if constexpr (QS == QS_Q23) s[2] = a6[0];
  }
}

// scale of sum (F^2)^q for one X-string: F = 2 W (x != 0) or W (x = 0)
template <int QS>
__device__ __forceinline__ double q_scale(int t, bool xzero, const QParams &qp) {
  if (xzero) return 1.0;
  if constexpr (QS == QS_Q2) return 16.0;
  if constexpr (QS == QS_Q23) return t == 0 ? 16.0 : 64.0;
  return pow_q_dev(4.0, qp.q[t]);
}

// ---------------------------------------------------------------------------------
// X-string bookkeeping for the two-pass engine.  Pass 1 pairs rows of the high index
// part, so the pairing bit jt of x must be >= PB.  For 1 <= x < 2^PB the kernel reads a
// copy of psi with bits j (the highest set bit of x) and n-1 swapped, on which the
// relabelled string xt = x ^ 2^j ^ 2^(n-1) has its pairing bit at n-1.  x = 0 is not
// handled by the two-pass kernel (its F is the plain transform of |psi|^2).
struct XInfo {
  uint64_t xt;  // effective x after the relabelling (pairing bit in the high part)
  int jt;       // pairing bit of xt
  int sw;       // relabelling: read the copy with bits sw and n-1 swapped (or -1)
  int active;   // Gray index inside the requested range and x != 0
  int zero = 0;  // x = 0 inside the range, built with the top-bit pairing (set by the caller)
};

__device__ __forceinline__ XInfo make_xinfo(uint64_t k, uint64_t k_end, int n, int pb) {
  XInfo xi;
  const uint64_t x = gray_code(k);
  xi.active = (k < k_end) && (x != 0);
  xi.zero = 0;
  xi.sw = -1;
  xi.xt = x;
  xi.jt = x ? 63 - __clzll((long long)x) : n - 1;
  if (x != 0 && xi.jt < pb) {
    xi.sw = xi.jt;
    xi.xt = (x ^ (1ull << xi.jt)) | (1ull << (n - 1));
    xi.jt = n - 1;
  }
  return xi;
}

// Pass 1: gather + build row rho of the (n-1)-bit index of x and transform its low PB
// bits.  The conj side a = psi(row rH) is loaded straight into the registers that will
// hold f; the partner row b = psi(row sH) goes to the warp's shared buffer through
// cp.async (no registers held while in flight), is read back permuted by the low bits
// of x, and the buffer is then reused for the transpose.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem_src) : "memory");
}
template <typename V>
__device__ __forceinline__ void cp_async_v(V *smem_dst, const V *gmem_src) {
  if constexpr (sizeof(V) == 16)
    cp_async16(smem_dst, gmem_src);
  else
    cp_async8(smem_dst, gmem_src);
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <int R, bool STAGE_B, typename V>
__device__ __forceinline__ void p1_build(V (&v)[R], const V *__restrict__ psi, const XInfo &xi, uint64_t rho, V *sm,
                                         int lane) {
  constexpr int PB = ilog2c(R) + 5;
  if (xi.zero) {
    // x = 0: f(r) = |psi(r)|^2 paired on the top bit (jt = n - 1),
    // h = (|a|^2 + |b|^2, |a|^2 - |b|^2) with a = psi(r), b = psi(r + 2^(n-1))
    const V *rowA = psi + (rho << PB);
    const V *rowB = rowA + (1ull << xi.jt);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint32_t e = (uint32_t)(i * 32 + lane);
      v[i] = zero_pair(ld_psi(rowA + e), ld_psi(rowB + e));
    }
    return;
  }
  const uint64_t rH = insert0(rho, xi.jt - PB);
  const uint64_t sH = rH ^ (xi.xt >> PB);
  const uint32_t xL = (uint32_t)(xi.xt & ((1ull << PB) - 1ull));
  const V *rowA = psi + (rH << PB);
  const V *rowB = psi + (sH << PB);
  if constexpr (STAGE_B) {
    // partner row, in natural order, into the shared buffer
#pragma unroll
    for (int i = 0; i < R; ++i) cp_async_v(sm + i * 32 + lane, rowB + i * 32 + lane);
    // conj side straight into registers
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = ld_psi(rowA + i * 32 + lane);
    cp_async_wait_all();
    __syncwarp();
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = conj_mul(v[i], sm[(uint32_t)(i * 32 + lane) ^ xL]);
    __syncwarp();  // the buffer is rewritten by the transpose
  } else {
    // both rows straight into registers (the partner permuted by the low bits of x)
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint32_t e = (uint32_t)(i * 32 + lane);
      v[i] = conj_mul(ld_psi(rowA + e), ld_psi(rowB + (e ^ xL)));
    }
  }
}

// Ring layout of one X-string's intermediate (2^(n-1) complex): tile-major,
//   inter_x[t * 2^(HI+LOGC) + row * C + c]  for pass-2 tile t, row, column c < C,
// so that a pass-2 tile is one contiguous 2^PB-element block and pass 1 writes whole
// 32-byte sectors (C >= 2).
// Hook run by every lane right before a pass-1 unit's first global store (the stage
// kernels wait there for the previous stage); the default does nothing.
struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};

template <int R, int HI, bool STAGE_B, typename V, typename Pre = NoHook>
__device__ __forceinline__ void p1_unit(const V *__restrict__ psi, const XInfo &xi, uint64_t rho,
                                        V *__restrict__ inter_x, V *sm, int lane, const Pre &pre = Pre()) {
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5, LOGC = PB - HI;
  V v[R];
  p1_build<R, STAGE_B>(v, psi, xi, rho, sm, lane);
  reg_wht<R, 0, LOGR>(v);  // element bits 5 .. PB-1
  transpose_ab<R>(v, sm, lane);
  reg_wht<R, 0, 5>(v);  // element bits 0 .. 4
  pre();
  // register i of lane l holds element k = R l + i; it is stored at position p = 32 i + l
  // of the row (any fixed relabelling of k is invisible to the moment sums)
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const uint32_t p = (uint32_t)(i * 32 + lane);
    const uint32_t t = p >> LOGC, c = p & ((1u << LOGC) - 1u);
    __stcg(inter_x + (((size_t)t << (HI + LOGC)) + (rho << LOGC) + c), v[i]);
  }
}

// ---------------------------------------------------------------------------------
// Pass-1 output through the tensor-memory-access unit.  The row's 2^PB positions land in
// 2^PB / C different pass-2 tiles, C positions each (C = 2 at n = 20): a warp-wide
// st.global of them touches 16 cache lines per instruction.  Instead the warp writes the
// row to its shared buffer in position order (conflict-free) and one thread issues
// tensor stores that scatter it to the tile-major ring (no multicast; the ring is this
// GPU's memory).  The 4-D tensor view of the ring, in scalars: d0 = the 2C scalars of a
// tile row, d1 = the 2^HI rows, d2 = the 2^PB / C tiles, d3 = the 2X (slot, X-string)
// pairs; boxes are {b0, 1, b2, 1}.
struct TmaGeom {
  int box0;  // scalars per box along d0 (2C, or 256 when 2C > 256)
  int nb0;   // boxes along d0 per tile (2C / box0)
  int box2;  // tiles per box (1 when nb0 > 1)
  int nb2;   // box groups along the tiles
  int C;     // positions per tile row
};

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_store_4d(const void *tmap, const void *smem_src, int c0, int c1, int c2, int c3) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_src);
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(tmap),
               "r"(s), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the shared-memory source of every committed store has been read
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// every committed store has completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// As p1_unit, with the row leaving through the warp's shared buffer and tensor stores.
// The caller waits for the stores to have read the buffer (bulk_wait_read_all on lane 0,
// then __syncwarp) before the buffer's next use.
template <int R, int HI, bool TM, typename V, typename Pre = NoHook, typename Ready = NoHook>
__device__ __forceinline__ void p1_unit_tma(const V *__restrict__ psi, const XInfo &xi, uint64_t rho, V *sm, int lane,
                                            const void *tmap, const TmaGeom &g, int xcoord, uint32_t ta,
                                            const Pre &pre = Pre(), const Ready &ready = Ready()) {
  constexpr int LOGR = ilog2c(R);
  V v[R];
  p1_build<R, false>(v, psi, xi, rho, sm, lane);  // registers only (no shared memory)
  reg_wht<R, 0, LOGR>(v);
  ready();  // the shared buffer is free from here on
#ifdef HM_TMEM_EXCHANGE
  if constexpr (TM) {
    static_assert(R == 32, "the TMEM exchanges are generated for 32 values per lane");
    tmem_row(v, ta);
  } else {
    transpose_ab<R>(v, sm, lane);
  }
#else
  (void)ta;
  transpose_ab<R>(v, sm, lane);
#endif
  reg_wht<R, 0, 5>(v);
  // register i of lane l holds element k = R l + i, kept at position p = 32 i + l
#pragma unroll
  for (int i = 0; i < R; ++i) sm[i * 32 + lane] = v[i];
  fence_proxy_async_smem();
  __syncwarp();
  pre();
  if (lane == 0) {
    for (int b2 = 0; b2 < g.nb2; ++b2)
      for (int b0 = 0; b0 < g.nb0; ++b0)
        tma_store_4d(tmap, sm + (size_t)b2 * g.box2 * g.C + (size_t)b0 * (g.box0 / 2), b0 * g.box0, (int)rho,
                     b2 * g.box2, xcoord);
    bulk_commit();
  }
}

// Pass 2: tile of 2^HI rows x C = 2^(PB-HI) positions of one X-string's intermediate
// (one contiguous block); transform over the row bits, then per-lane moments.
template <int R, int HI, int QS, bool TM = false, typename V, typename Ready = NoHook>
__device__ __forceinline__ void p2_unit(const V *__restrict__ tile_ptr, V *sm, int lane, double *s,
                                        const QParams &qp, uint32_t ta = 0, const Ready &ready = Ready()) {
  (void)ta;
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5, LOGC = PB - HI;
  static_assert(HI >= 1 && HI <= PB, "pass-2 bits out of range");
  V v[R];
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = __ldcg(tile_ptr + i * 32 + lane);
  if constexpr (LOGC >= 5) {
    reg_wht<R, LOGC - 5, LOGR>(v);
    ready();
#ifdef HM_TMEM_EXCHANGE
  } else if constexpr (TM && R == 32) {
    reg_wht<R, 0, LOGR>(v);
    ready();
    tmem_tile<HI>(v, ta);
    reg_wht<R, 0, 5 - LOGC>(v);
#endif
  } else {
    reg_wht<R, 0, LOGR>(v);
    ready();
    transpose_ab<R>(v, sm, lane);
    reg_wht<R, LOGC, 5>(v);
  }
  lane_moments<R, QS>(v, s, qp, sm, lane);
}

}  // namespace hm
