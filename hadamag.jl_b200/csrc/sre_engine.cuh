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
// for x != 0; the caller applies the 4 / 4^q scale).  FP64: plain sums in a fixed
// order.  FP32: eight interleaved float accumulators per sum, combined pairwise, then
// promoted to double.
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

template <int R, int QS>
__device__ __forceinline__ void lane_moments(const double2 (&v)[R], double *s, const QParams &qp, double2 *sm,
                                             int lane) {
  if constexpr (QS == QS_GEN) {
#pragma unroll
    for (int i = 0; i < R; ++i) sm[lane + 32 * i] = v[i];
    lane_moments_gen<R>(sm, lane, s, qp);
    __syncwarp();
    return;
  } else {
    double a2 = 0.0, a4 = 0.0, a6 = 0.0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const double f = c ? v[i].y : v[i].x;
        const double y = f * f;
        a2 += y;
        a4 = fma(y, y, a4);
        if constexpr (QS == QS_Q23) a6 = fma(y * y, y, a6);
      }
    }
    s[0] = a2;
    s[1] = a4;
    if constexpr (QS == QS_Q23) s[2] = a6;
  }
}

template <int R, int QS>
__device__ __forceinline__ void lane_moments(const float2 (&v)[R], double *s, const QParams &qp, float2 *sm,
                                             int lane) {
  if constexpr (QS == QS_GEN) {
#pragma unroll
    for (int i = 0; i < R; ++i) sm[lane + 32 * i] = v[i];
    lane_moments_gen<R>(sm, lane, s, qp);
    __syncwarp();
    return;
  } else {
    constexpr int NA = 8;
    float a2[NA], a4[NA], a6[NA];
#pragma unroll
    for (int t = 0; t < NA; ++t) a2[t] = a4[t] = a6[t] = 0.f;
#pragma unroll
    for (int i = 0; i < R; ++i) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const float f = c ? v[i].y : v[i].x;
        const float y = f * f;
        const int t = (2 * i + c) % NA;
        a2[t] += y;
        a4[t] = fmaf(y, y, a4[t]);
        if constexpr (QS == QS_Q23) a6[t] = fmaf(y * y, y, a6[t]);
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
    s[0] = (double)a2[0];
    s[1] = (double)a4[0];
    if constexpr (QS == QS_Q23) s[2] = (double)a6[0];
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
// X-string bookkeeping for the two-pass engine
struct XInfo {
  uint64_t xt;  // effective x after the relabelling (pairing bit in the high part)
  int jt;       // pairing bit of xt
  int sw;       // relabelling: swap bit sw with bit n-1 (or -1)
  int zero;     // x == 0
  int active;   // Gray index inside the requested range
};

__device__ __forceinline__ XInfo make_xinfo(uint64_t k, uint64_t k_end, int n, int pb) {
  XInfo xi;
  xi.active = k < k_end;
  const uint64_t x = gray_code(k);
  xi.zero = (x == 0);
  xi.sw = -1;
  if (x == 0) {
    xi.xt = 1ull << (n - 1);
    xi.jt = n - 1;
  } else {
    const int j = 63 - __clzll((long long)x);
    if (j >= pb) {
      xi.xt = x;
      xi.jt = j;
    } else {
      xi.xt = (x ^ (1ull << j)) | (1ull << (n - 1));
      xi.jt = n - 1;
      xi.sw = j;
    }
  }
  return xi;
}

// Pass 1: gather + build row rho of the (n-1)-bit index of x, transform its low PB
// bits, store it in layout-A order (position p = 32 i + l for the value of register i
// of lane l, i.e. element k = R l + i).
template <int R, bool ZERO, bool SWAP, typename V>
__device__ __forceinline__ void p1_build(V (&v)[R], const V *__restrict__ psi, int n, const XInfo &xi,
                                         uint64_t rho, int lane) {
  constexpr int PB = ilog2c(R) + 5;
  const uint64_t rH = insert0(rho, xi.jt - PB);
  const uint64_t sH = rH ^ (xi.xt >> PB);
  const uint32_t xL = (uint32_t)(xi.xt & ((1ull << PB) - 1ull));
  const uint64_t baseA = rH << PB, baseB = sH << PB;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const uint32_t e = (uint32_t)(i * 32 + lane);
    uint64_t ra = baseA | e, rb = baseB | (e ^ xL);
    if (SWAP) {
      ra = swap_bits(ra, xi.sw, n - 1);
      rb = swap_bits(rb, xi.sw, n - 1);
    }
    const V a = ld_psi(psi + ra), b = ld_psi(psi + rb);
    v[i] = ZERO ? zero_pair(a, b) : conj_mul(a, b);
  }
}

template <int R, typename V>
__device__ __forceinline__ void p1_unit(const V *__restrict__ psi, int n, const XInfo &xi, uint64_t rho,
                                        V *__restrict__ out_row, V *sm, int lane) {
  constexpr int LOGR = ilog2c(R);
  V v[R];
  if (xi.zero)
    p1_build<R, true, false>(v, psi, n, xi, rho, lane);
  else if (xi.sw >= 0)
    p1_build<R, false, true>(v, psi, n, xi, rho, lane);
  else
    p1_build<R, false, false>(v, psi, n, xi, rho, lane);
  reg_wht<R, 0, LOGR>(v);  // element bits 5 .. PB-1
  transpose_ab<R>(v, sm, lane);
  reg_wht<R, 0, 5>(v);  // element bits 0 .. 4
#pragma unroll
  for (int i = 0; i < R; ++i) __stcg(out_row + i * 32 + lane, v[i]);
}

// Pass 2: tile of 2^HI rows x C = 2^(PB-HI) consecutive positions of one X-string's
// intermediate; transform over the row bits, then per-lane moments.
template <int R, int HI, int QS, typename V>
__device__ __forceinline__ void p2_unit(const V *__restrict__ inter_x, uint32_t tile, V *sm, int lane, double *s,
                                        const QParams &qp) {
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5, LOGC = PB - HI, C = 1 << LOGC;
  static_assert(HI >= 1 && HI <= PB, "pass-2 bits out of range");
  V v[R];
  const uint32_t p0 = tile * C;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const uint32_t e = (uint32_t)(i * 32 + lane);
    const uint32_t row = e >> LOGC, c = e & (C - 1);
    v[i] = __ldcg(inter_x + (size_t)row * (32 * R) + p0 + c);
  }
  if constexpr (LOGC >= 5) {
    reg_wht<R, LOGC - 5, LOGR>(v);
  } else {
    reg_wht<R, 0, LOGR>(v);
    transpose_ab<R>(v, sm, lane);
    reg_wht<R, LOGC, 5>(v);
  }
  lane_moments<R, QS>(v, s, qp, sm, lane);
}

}  // namespace hm
