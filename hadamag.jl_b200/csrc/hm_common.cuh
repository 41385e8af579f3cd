// hm_common.cuh -- device helpers shared by the hadamag_b200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hm {

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }

// Complex vector type per precision.
template <typename T> struct VT;
template <> struct VT<double> { typedef double2 V; };
template <> struct VT<float> { typedef float2 V; };

template <typename V>
__device__ __forceinline__ V v_add(V a, V b) {
  V r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename V>
__device__ __forceinline__ V v_sub(V a, V b) {
  V r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
#ifndef HM_NO_F32X2
// FP32 complex values: one packed two-lane instruction (add/sub.rn.f32x2, sm_100) per
// butterfly output instead of two; per lane the same round-to-nearest result as a + b.
template <>
__device__ __forceinline__ float2 v_add<float2>(float2 a, float2 b) {
  unsigned long long ra, rb, rc;
  asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(rc) : "l"(ra), "l"(rb));
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(rc));
  return r;
}
template <>
__device__ __forceinline__ float2 v_sub<float2>(float2 a, float2 b) {
  unsigned long long ra, rb, rc;
  asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rc) : "l"(ra), "l"(rb));
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(rc));
  return r;
}
#endif

// Double-double accumulator (Knuth TwoSum on every addition).  Sums of partial
// results land within ~1e-30 relative of the exact sum, so the final rounding to
// double does not depend on the order in which partials arrive.
struct dd {
  double hi, lo;
};
__device__ __forceinline__ void dd_add(dd &a, double b) {
  double s = a.hi + b;
  double bb = s - a.hi;
  double err = (a.hi - (s - bb)) + (b - bb);
  a.hi = s;
  a.lo += err;
}
__device__ __forceinline__ void dd_add_dd(dd &a, const dd &b) {
  double s = a.hi + b.hi;
  double bb = s - a.hi;
  double err = (a.hi - (s - bb)) + (b.hi - bb);
  double lo = a.lo + b.lo + err;
  double hi = s + lo;
  a.lo = lo - (hi - s);
  a.hi = hi;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ uint64_t gray_code(uint64_t k) { return k ^ (k >> 1); }

// value with a zero bit inserted at position p
__device__ __forceinline__ uint64_t insert0(uint64_t v, int p) {
  const uint64_t lo = v & ((1ull << p) - 1ull);
  return ((v >> p) << (p + 1)) | lo;
}

// swap bits a and b of r
__device__ __forceinline__ uint64_t swap_bits(uint64_t r, int a, int b) {
  const uint64_t d = ((r >> a) ^ (r >> b)) & 1ull;
  return r ^ (d << a) ^ (d << b);
}

}  // namespace hm
