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
