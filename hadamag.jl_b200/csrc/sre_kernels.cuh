// sre_kernels.cuh -- exact-SRE kernels (fused single-warp sweep for n <= PB+1, and the
// persistent two-pass sweep for larger n) plus the deterministic double-double fold.
#pragma once
#include "sre_engine.cuh"

namespace hm {

struct SreArgs {
  const void *psi;   // V[2^n] (double2 or float2)
  const void *psi_sw[16];  // two-pass: psi with bits j and n-1 swapped, j < PB
  void *inter;       // two-pass ring: S batch slots x X strings x 2^(n-1) V
  double *partials;  // per warp: 2 * (1 + NQ) doubles (dd per sum)
  unsigned *ctrl;    // [0,1] 64-bit queue head, [2] error flag, [4, 4+S) pass-1 done, [4+S, 4+2S) pass-2 done,
                     // [4+2S, 4+2S+2) 64-bit sum of dependency-wait cycles, [+2, +4) 64-bit sum of CTA cycles
  uint64_t k_begin, k_end;
  long long nitems;     // queue length (CTA items)
  long long spin_limit; // clock cycles before a dependency wait gives up
  QParams qp;
  int n, X, S, nbatch;
  int upw;    // two-pass: warp units per warp per CTA item
  int flags;  // bit 1: every lane fences its stores before the completion signal
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
// per X-string); a CTA item is SRE_WARPS consecutive units (the same row of the batch's
// X-strings, so the state rows they gather are shared through L1).  P2(b) waits for
// all of P1(b); P1(b) waits for P2(b - S) to have released the slot.  Items are handed
// out in order by an atomic queue, so every awaited item is already owned by a running
// CTA: the waits always end (each is also bounded by spin_limit, after which the error
// flag stops every CTA).  Thread 0 fetches the next item while the warps work on the
// current one, then publishes the finished item with one fence and one counter update.
// CTAs per SM the register budget is sized for: FP64 keeps 32 complex (128 registers)
// of data per lane, FP32 half of that.
template <typename T> struct TwoPassOcc { static constexpr int value = sizeof(T) == 8 ? 2 : 4; };

template <typename T, int R, int HI, int QS>
__global__ void __launch_bounds__(SRE_WARPS * 32, TwoPassOcc<T>::value) k_sre_2pass(SreArgs a) {
  using V = typename VT<T>::V;
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5, NQ = QSet<QS>::NQ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long s_item[2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *sm = reinterpret_cast<V *>(smem_raw) + warp * (32 * R);
  const int gwarp = blockIdx.x * SRE_WARPS + warp;
  const V *psi = reinterpret_cast<const V *>(a.psi);
  V *inter = reinterpret_cast<V *>(a.inter);
  const int n = a.n;
  const uint64_t U = 1ull << HI;          // units per X-string per pass
  const uint64_t xlen = 1ull << (n - 1);  // intermediate length per X-string
  const long long K = (long long)((a.X * U) / (SRE_WARPS * a.upw));  // CTA items per pass per batch
  unsigned *err = a.ctrl + 2;
  unsigned *p1_done = a.ctrl + 4;
  unsigned *p2_done = a.ctrl + 4 + a.S;
  const unsigned per_pass = (unsigned)(a.X * U);
  unsigned long long *queue = reinterpret_cast<unsigned long long *>(a.ctrl);

  // item -> (pass, batch, index of the CTA item within the pass)
  auto decode = [&](long long item, int &pass, long long &b, long long &r) {
    if (item < K) {
      pass = 1;
      b = 0;
      r = item;
      return;
    }
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
  };
  // thread 0 only: wait until the item's inputs (pass 2) or its ring slot (pass 1) are
  // ready.  Counter values already observed are kept per slot, so repeated checks of a
  // satisfied dependency cost no L2 round trip.
  unsigned seen1[8], seen2[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) seen1[i] = seen2[i] = 0u;
  auto wait_cached = [&](unsigned *ctr, unsigned &seen, unsigned target) -> bool {
    if (seen >= target) return true;
    if (!wait_counter(ctr, target, err, a.spin_limit)) return false;
    seen = target;
    return true;
  };
  auto wait_deps = [&](long long item) -> bool {
    if (item >= a.nitems) return true;
    int pass;
    long long b, r;
    decode(item, pass, b, r);
    const int slot = (int)(b % a.S);
    const unsigned gen = (unsigned)(b / a.S);
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (i == slot) {
        if (pass == 2)
          ok = wait_cached(p1_done + i, seen1[i], (gen + 1) * per_pass);
        else if (b >= a.S)
          ok = wait_cached(p2_done + i, seen2[i], gen * per_pass);
      }
    return ok;
  };

  dd acc[NQ + 1];
#pragma unroll
  for (int t = 0; t <= NQ; ++t) acc[t] = dd{0.0, 0.0};

  long long t_start = clock64(), t_wait = 0;
  if (threadIdx.x == 0) {
    long long it = (long long)atomicAdd(queue, 1ull);
    if (!wait_deps(it)) it = a.nitems;
    s_item[0] = it;
  }
  __syncthreads();
  for (int j = 0;; ++j) {
    const long long item = s_item[j & 1];
    if (item >= a.nitems) break;
    long long next = 0;
    if (threadIdx.x == 0) next = (long long)atomicAdd(queue, 1ull);  // latency hidden by the work below
    int pass;
    long long b, r;
    decode(item, pass, b, r);
    const int slot = (int)(b % a.S);
    for (int t = 0; t < a.upw; ++t) {
      // at each step the CTA's warps take consecutive units: the same rows of the
      // batch's X-strings, whose state rows they share through L1
      const uint64_t u = ((uint64_t)r * a.upw + t) * SRE_WARPS + warp;  // warp unit within the pass
      const int xs = (int)(u % a.X);                                     // X-string slot in the batch
      const uint64_t sub = u / a.X;                                      // row (pass 1) or tile (pass 2)
      const uint64_t k = a.k_begin + (uint64_t)b * a.X + xs;
      V *inter_x = inter + ((size_t)slot * a.X + xs) * xlen;
      const XInfo xi = make_xinfo(k, a.k_end, n, PB);
      if (pass == 1) {
        if (xi.active) {
          const V *src = xi.sw < 0 ? psi : reinterpret_cast<const V *>(a.psi_sw[xi.sw]);
          if (a.flags & 16)
            p1_unit<R, HI, true>(src, xi, sub, inter_x, sm, lane);
          else
            p1_unit<R, HI, false>(src, xi, sub, inter_x, sm, lane);
        }
      } else if (xi.active) {
        double s[NQ + 1];
        p2_unit<R, HI, QS>(inter_x + (sub << PB), sm, lane, s, a.qp);
        s[0] = 4.0 * s[0];
#pragma unroll
        for (int q = 0; q < NQ; ++q) s[1 + q] *= q_scale<QS>(q, false, a.qp);
#pragma unroll
        for (int q = 0; q <= NQ; ++q) dd_add(acc[q], warp_sum(s[q]));
      }
    }
    __syncthreads();  // every warp of the CTA finished its unit of this item
    if (threadIdx.x == 0) {
      unsigned *ctr = (pass == 1 ? p1_done : p2_done) + slot;
      const unsigned inc = (unsigned)(SRE_WARPS * a.upw);
      if (a.flags & 4) {
        red_release_gpu_add(ctr, inc);
      } else if (a.flags & 8) {
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        atomicAdd(ctr, inc);
      } else {
        __threadfence();
        atomicAdd(ctr, inc);
      }
      const long long w0 = clock64();
      if (*(volatile unsigned *)err || !wait_deps(next)) next = a.nitems;
      t_wait += clock64() - w0;
      s_item[(j + 1) & 1] = next;
    }
    __syncthreads();
  }
  if (lane == 0) write_partials<NQ>(a.partials, gwarp, acc);
  if (threadIdx.x == 0) {
    unsigned long long *st = reinterpret_cast<unsigned long long *>(a.ctrl + 4 + 2 * a.S);
    atomicAdd(st, (unsigned long long)t_wait);
    atomicAdd(st + 1, (unsigned long long)(clock64() - t_start));
  }
}

// ---------------------------------------------------------------------------------
// Deterministic fold of per-warp double-double partials: out[2t], out[2t+1] = dd of sum t.
__global__ void k_fold_partials(const double *__restrict__ partials, int nwarps, int nsum, double *out);

// psi (double2) -> float2 copy for the FP32 path
__global__ void k_psi_to_f32(const double2 *__restrict__ in, float2 *__restrict__ out, uint64_t len);

// copies of psi with bits j and n-1 swapped, j = 0 .. nj-1 (out holds nj states back to back)
template <typename V>
__global__ void k_psi_swapped(const V *__restrict__ in, V *__restrict__ out, int n, int nj) {
  const uint64_t len = 1ull << n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len * nj;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const int j = (int)(i >> n);
    const uint64_t r = i & (len - 1);
    out[i] = in[swap_bits(r, j, n - 1)];
  }
}

}  // namespace hm
