// sre_kernels.cuh -- exact-SRE kernels (fused single-warp sweep for n <= PB+1, and the
// persistent two-pass sweep for larger n) plus the deterministic double-double fold.
#pragma once
#include "sre_engine.cuh"

namespace hm {

struct SreArgs {
  const void *psi;   // V[2^n] (double2 or float2)
  void *inter;       // two-pass ring: S batch slots x X strings x 2^(n-1) V
  double *partials;  // per warp: 2 * (1 + NQ) doubles (dd per sum)
  unsigned *ctrl;    // [0,1] 64-bit queue head, [2] error flag, [4, 4+S) pass-1 done, [4+S, 4+2S) pass-2 done
  uint64_t k_begin, k_end;
  long long nitems;     // queue length (CTA items)
  long long spin_limit; // clock cycles before a dependency wait gives up
  QParams qp;
  int n, X, S, nbatch;
};

constexpr int SRE_WARPS = 4;  // warps per CTA in the two-pass kernel
constexpr int FUSED_WARPS = 4;

template <int NQ>
__device__ __forceinline__ void write_partials(double *partials, int gwarp, const dd *acc) {
#pragma unroll
  for (int t = 0; t <= NQ; ++t) {
    partials[(size_t)gwarp * 2 * (NQ + 1) + 2 * t] = acc[t].hi;
    partials[(size_t)gwarp * 2 * (NQ + 1) + 2 * t + 1] = acc[t].lo;
  }
}

// ---------------------------------------------------------------------------------
// Fused sweep, n - 1 = NB <= PB element bits: one warp holds 2^(PB - NB) X-strings
// (consecutive Gray indices), builds, transforms and reduces them without leaving the SM.
template <typename T, int R, int NB, int QS>
__global__ void __launch_bounds__(FUSED_WARPS * 32) k_sre_fused(SreArgs a) {
  using V = typename VT<T>::V;
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5, NQ = QSet<QS>::NQ;
  constexpr bool LANE_UNIFORM = NB >= LOGR;  // in layout B each lane holds one X-string
  static_assert(NB <= PB, "fused kernel covers n - 1 <= PB");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *sm = reinterpret_cast<V *>(smem_raw) + (threadIdx.x >> 5) * (32 * R);
  const int lane = threadIdx.x & 31;
  const int gwarp = blockIdx.x * FUSED_WARPS + (threadIdx.x >> 5);
  const int nwarps = gridDim.x * FUSED_WARPS;
  const V *psi = reinterpret_cast<const V *>(a.psi);
  constexpr uint64_t XPW = 1ull << (PB - NB);
  const uint64_t ngroups = (a.k_end - a.k_begin + XPW - 1) / XPW;
  dd acc[NQ + 1];
#pragma unroll
  for (int t = 0; t <= NQ; ++t) acc[t] = dd{0.0, 0.0};

  for (uint64_t g = gwarp; g < ngroups; g += nwarps) {
    const uint64_t kbase = a.k_begin + g * XPW;
    V v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint32_t e = (uint32_t)(i * 32 + lane);
      const uint64_t xl = e >> NB, rp = e & ((1u << NB) - 1u);
      const uint64_t k = kbase + xl;
      V f;
      f.x = 0;
      f.y = 0;
      if (k < a.k_end) {
        const uint64_t x = gray_code(k);
        if (x == 0) {
          f = zero_pair(ld_psi(psi + rp), ld_psi(psi + rp + (1ull << NB)));
        } else {
          const int j = 63 - __clzll((long long)x);
          const uint64_t r = insert0(rp, j);
          f = conj_mul(ld_psi(psi + r), ld_psi(psi + (r ^ x)));
          if (!LANE_UNIFORM) {
            f.x += f.x;
            f.y += f.y;
          }
        }
      }
      v[i] = f;
    }
    if constexpr (NB > 5) reg_wht<R, 0, NB - 5>(v);
    transpose_ab<R>(v, sm, lane);
    reg_wht<R, 0, (NB < 5 ? NB : 5)>(v);
    double s[NQ + 1];
    lane_moments<R, QS>(v, s, a.qp, sm, lane);
    if (LANE_UNIFORM) {
      const uint64_t k = kbase + (((uint64_t)lane * R) >> NB);
      const bool act = k < a.k_end;
      const bool xz = gray_code(k) == 0;
      s[0] = act ? (xz ? s[0] : 4.0 * s[0]) : 0.0;
#pragma unroll
      for (int t = 0; t < NQ; ++t) s[1 + t] = act ? s[1 + t] * q_scale<QS>(t, xz, a.qp) : 0.0;
    }
#pragma unroll
    for (int t = 0; t <= NQ; ++t) dd_add(acc[t], warp_sum(s[t]));
  }
  if (lane == 0) write_partials<NQ>(a.partials, gwarp, acc);
}

// ---------------------------------------------------------------------------------
// Two-pass persistent sweep.  Work is a queue of CTA items in a fixed order
//   P1(0), [P1(1), P2(0)], [P1(2), P2(1)], ..., [P1(B-1), P2(B-2)], P2(B-1)
// where batch b holds X consecutive Gray indices and its intermediate lives in ring
// slot b % S.  Each pass of a batch is X * U warp units (U = 2^HI rows, resp. tiles,
// per X-string), grouped SRE_WARPS per CTA item.  P2(b) waits for all of P1(b); P1(b)
// waits for P2(b - S) to have released the slot.  Items are handed out in order by an
// atomic queue, so every awaited item is already owned by a running CTA: the waits
// always end (each is also bounded by spin_limit and then raises the error flag).
template <typename T, int R, int HI, int QS>
__global__ void __launch_bounds__(SRE_WARPS * 32) k_sre_2pass(SreArgs a) {
  using V = typename VT<T>::V;
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5, NQ = QSet<QS>::NQ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long s_item;
  __shared__ int s_ok;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *sm = reinterpret_cast<V *>(smem_raw) + warp * (32 * R);
  const int gwarp = blockIdx.x * SRE_WARPS + warp;
  const V *psi = reinterpret_cast<const V *>(a.psi);
  V *inter = reinterpret_cast<V *>(a.inter);
  const int n = a.n;
  const uint64_t U = 1ull << HI;                        // units per X-string per pass
  const uint64_t xlen = 1ull << (n - 1);                // intermediate length per X-string
  const long long K = (long long)((a.X * U) / SRE_WARPS);  // CTA items per pass per batch
  unsigned *err = a.ctrl + 2;
  unsigned *p1_done = a.ctrl + 4;
  unsigned *p2_done = a.ctrl + 4 + a.S;
  const unsigned per_pass = (unsigned)(a.X * U);

  dd acc[NQ + 1];
#pragma unroll
  for (int t = 0; t <= NQ; ++t) acc[t] = dd{0.0, 0.0};

  for (;;) {
    if (threadIdx.x == 0) {
      long long it = (long long)atomicAdd(reinterpret_cast<unsigned long long *>(a.ctrl), 1ull);
      if (*(volatile unsigned *)err) it = a.nitems;  // another CTA gave up: stop everyone
      s_item = it;
    }
    __syncthreads();
    const long long item = s_item;
    if (item >= a.nitems) break;
    // decode the item
    int pass;
    long long b, r;
    if (item < K) {
      pass = 1;
      b = 0;
      r = item;
    } else {
      const long long it = item - K;
      const long long t = 1 + it / (2 * K);
      const long long rr = it % (2 * K);
      if (t >= a.nbatch) {
        pass = 2;
        b = a.nbatch - 1;
        r = rr;
      } else if (rr < K) {
        pass = 1;
        b = t;
        r = rr;
      } else {
        pass = 2;
        b = t - 1;
        r = rr - K;
      }
    }
    const int slot = (int)(b % a.S);
    const unsigned gen = (unsigned)(b / a.S);
    if (threadIdx.x == 0) {
      bool ok = true;
      if (pass == 2)
        ok = wait_counter(p1_done + slot, (gen + 1) * per_pass, err, a.spin_limit);
      else if (b >= a.S)
        ok = wait_counter(p2_done + slot, gen * per_pass, err, a.spin_limit);
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) break;
    const uint64_t u = (uint64_t)r * SRE_WARPS + warp;  // warp unit within the pass
    const int xs = (int)(u % a.X);                        // X-string slot in the batch
    const uint64_t sub = u / a.X;                         // row (pass 1) or tile (pass 2)
    const uint64_t k = a.k_begin + (uint64_t)b * a.X + xs;
    V *inter_x = inter + ((size_t)slot * a.X + xs) * xlen;
    const XInfo xi = make_xinfo(k, a.k_end, n, PB);
    if (pass == 1) {
      if (xi.active) p1_unit<R>(psi, n, xi, sub, inter_x + sub * (32 * R), sm, lane);
      __threadfence();
      __syncwarp();
      if (lane == 0) red_release_gpu_add(p1_done + slot, 1u);
    } else {
      if (xi.active) {
        double s[NQ + 1];
        p2_unit<R, HI, QS>(inter_x, (uint32_t)sub, sm, lane, s, a.qp);
        s[0] = xi.zero ? s[0] : 4.0 * s[0];
#pragma unroll
        for (int t = 0; t < NQ; ++t) s[1 + t] *= q_scale<QS>(t, xi.zero, a.qp);
#pragma unroll
        for (int t = 0; t <= NQ; ++t) dd_add(acc[t], warp_sum(s[t]));
      }
      __syncwarp();
      if (lane == 0) red_release_gpu_add(p2_done + slot, 1u);
    }
    __syncthreads();  // s_item / s_ok are rewritten by the next dequeue
  }
  if (lane == 0) write_partials<NQ>(a.partials, gwarp, acc);
}

// ---------------------------------------------------------------------------------
// Deterministic fold of per-warp double-double partials: out[2t], out[2t+1] = dd of sum t.
__global__ void k_fold_partials(const double *__restrict__ partials, int nwarps, int nsum, double *out);

// psi (double2) -> float2 copy for the FP32 path
__global__ void k_psi_to_f32(const double2 *__restrict__ in, float2 *__restrict__ out, uint64_t len);

}  // namespace hm
