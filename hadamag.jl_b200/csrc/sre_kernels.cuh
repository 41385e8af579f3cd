// sre_kernels.cuh -- exact-SRE kernels (fused single-warp sweep for n <= PB+1, and the
// two-pass stage kernels for larger n) plus the deterministic double-double fold.
#pragma once
#include <cuda.h>  // CUtensorMap

#include "sre_engine.cuh"

namespace hm {

struct SreArgs {
  const void *psi;   // V[2^n] (double2 or float2)
  double *partials;  // per warp: 2 * (1 + NQ) doubles (dd per sum)
  uint64_t k_begin, k_end;
  QParams qp;
  int n;
};

constexpr int SRE_WARPS = 4;  // warps per CTA in the two-pass stage kernels
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
// The state is always read in FP64 and f = conj(psi(r)) psi(r ^ x) is formed in FP64;
// the FP32 variant rounds f, not psi, so that its error stays second order.
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
  const double2 *psi = reinterpret_cast<const double2 *>(a.psi);
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
      double2 f = make_double2(0.0, 0.0);
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
      v[i].x = (T)f.x;
      v[i].y = (T)f.y;
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
// Two-pass sweep as a sequence of stage kernels.  Stage t runs pass 1 of batch t and
// pass 2 of batch t - 1 (independent work: the kernel boundary is the only dependency),
// with batch b's intermediate in ring slot b % 2.  Every warp walks a fixed round-robin
// share of the stage's units and adds its moment sums into its own double-double slot,
// so the result does not depend on scheduling.  A block of stages is captured once as a
// CUDA graph and replayed: node `node` of the graph runs stage base + node, with `base`
// in device memory, advanced by a one-thread kernel at the end of every replay.
// The stage nodes are chained by programmatic dependent launch: stage t + 1 may start on
// the SMs that stage t has already left.  It then runs the reads of psi and the
// butterflies of its first pass-1 units, and waits for stage t to finish (and its memory
// to be visible) only before its first access that depends on stage t: a ring store
// (the slot that stage t's pass 2 reads), a ring load, the moment-slot update.
// CTAs per SM of the stage kernels: FP64 keeps 32 complex (128 registers) of data per
// lane and runs at 255 registers (8 warps / SM), FP32 at 128 registers (16 warps / SM)
template <typename T> struct StageOcc { static constexpr int value = sizeof(T) == 8 ? 2 : 4; };

struct StageArgs {
  CUtensorMap tmap;    // tensor view of the ring for the pass-1 stores (valid when tma)
  const void *psi;
  const void *psi_sw[16];
  void *ring;          // 2 slots x X strings x 2^(n-1) V
  double *slots;       // per warp: 2 (1 + NQ) doubles
  unsigned *stage;     // [0] stage index of node 0 of the current graph replay
  uint64_t k_begin, k_end;
  QParams qp;
  TmaGeom g;
  int n, X, nbatch, tma;
  int node;            // position of this launch in the captured graph
};

// wait for the preceding grid (programmatic dependent launch); immediate otherwise
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// let the next grid in the stream be scheduled before this one finishes
__device__ __forceinline__ void allow_next_grid() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// one thread: advance the stage base past the stages of the replay that just ran
__global__ void k_stage_advance(unsigned *stage, unsigned count);

template <typename T, int R, int HI, int QS>
__global__ void __launch_bounds__(SRE_WARPS * 32, StageOcc<T>::value)
    k_sre_stage(const __grid_constant__ StageArgs a) {
  using V = typename VT<T>::V;
  constexpr int LOGR = ilog2c(R), PB = LOGR + 5, NQ = QSet<QS>::NQ;
  // the tensor stores read the per-warp buffers: keep them 1024-byte aligned
  extern __shared__ __align__(1024) unsigned char smem_stage[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *sm = reinterpret_cast<V *>(smem_stage) + warp * (32 * R);
  allow_next_grid();
  // the base only changes between replays, after every node of the replay has finished
  const long long t = (long long)*(volatile unsigned *)a.stage + a.node;
  if (t > a.nbatch) return;  // padding stages of the last graph replay
#ifdef HM_TMEM_EXCHANGE
  // TMEM for the lane <-> register exchanges (the whole CTA takes part; no return below)
  __shared__ uint32_t tmem_slot;
  const uint32_t tmem_base = tmem_cta_alloc(&tmem_slot, TmemCols<T>::value);
  const uint32_t ta = tmem_warp_addr(tmem_base);
  constexpr bool TM = true;
#else
  const uint32_t ta = 0;
  constexpr bool TM = false;
#endif
  const int gwarp = blockIdx.x * SRE_WARPS + warp;
  const int nwarps = gridDim.x * SRE_WARPS;
  const V *psi = reinterpret_cast<const V *>(a.psi);
  V *ring = reinterpret_cast<V *>(a.ring);
  const int n = a.n;
  const uint64_t U = 1ull << HI;
  const uint64_t xlen = 1ull << (n - 1);
  const long long per = (long long)a.X * (long long)U;
  const long long n2 = (t >= 1) ? per : 0;              // pass-2 units of batch t-1
  const long long n1 = (t < a.nbatch) ? per : 0;        // pass-1 units of batch t
  // FP64 keeps the moment sums per lane and reduces them across the warp once per stage
  // (1-3 % faster on B200); FP32, at half the registers, sums each unit across the warp
  // (per-lane accumulators cost it 2 %).  Both orders are fixed.
  constexpr bool LANE_ACC = sizeof(T) == 8;
  dd acc[NQ + 1];
#pragma unroll
  for (int q = 0; q <= NQ; ++q) acc[q] = dd{0.0, 0.0};
  // Unit order per warp: one pass-1 unit first (its psi reads and butterflies overlap the
  // previous stage's tail), then the pass-2 units (they read the previous stage's rows
  // while those are still in L2), then the other pass-1 units.  Measured on B200 against
  // pass 1 first / pass 2 first: -5 % to -12 % at n = 18, 20, 21 in FP64.
  auto pre = [] { wait_prior_grid(); };
  const long long nfirst = n1 < nwarps ? n1 : nwarps;
  for (long long u = gwarp; u < n1 + n2; u += nwarps) {
    const bool p2 = u >= nfirst && u < nfirst + n2;
    const long long r = p2 ? u - nfirst : (u < nfirst ? u : u - n2);
    const long long b = p2 ? t - 1 : t;
    const int xs = (int)(r % a.X);
    const uint64_t sub = (uint64_t)(r / a.X);
    const uint64_t k = a.k_begin + (uint64_t)b * a.X + xs;
    V *inter_x = ring + ((size_t)(b & 1) * a.X + xs) * xlen;
    XInfo xi = make_xinfo(k, a.k_end, n, PB);
    xi.zero = k < a.k_end && xi.xt == 0;  // x = 0 (Gray index 0): built with the top-bit pairing
    if (!xi.active && !xi.zero) continue;
    // the previous unit's tensor stores must have read the shared buffer before this unit
    // writes it: waited for right before the unit's first shared-memory access, so that
    // the stores' read overlaps this unit's global loads and first butterflies
    auto ready = [&] {
      if (a.tma) {
        if (lane == 0) bulk_wait_read_all();
        __syncwarp();
      }
    };
    if (!p2) {
      const V *src = xi.sw < 0 ? psi : reinterpret_cast<const V *>(a.psi_sw[xi.sw]);
      if (a.tma)
        p1_unit_tma<R, HI, TM>(src, xi, sub, sm, lane, &a.tmap, a.g, (int)((b & 1) * a.X + xs), ta, pre, ready);
      else
        p1_unit<R, HI, false>(src, xi, sub, inter_x, sm, lane, pre);
    } else {
      double s[NQ + 1];
      wait_prior_grid();
      p2_unit<R, HI, QS, TM>(inter_x + (sub << PB), sm, lane, s, a.qp, ta, ready);
      // The tile is dead once read (its slot is rewritten by pass 1 two stages later, in
      // another launch): drop its L2 lines without writing them back to DRAM.  The next
      // write to the slot comes after griddepcontrol.wait on the launch in between, which
      // returns once this launch has finished and its memory operations are performed.
      // Within one launch a discard is NOT ordered by release/acquire on B200: the queue
      // sweep, whose slots are rewritten inside the same launch, lost data when it
      // discarded its tiles, so it does not.
      {
        const char *tb = reinterpret_cast<const char *>(inter_x + (sub << PB));
        constexpr int LINES = (int)(32 * R * sizeof(V) / 128);
#pragma unroll
        for (int ln = lane; ln < LINES; ln += 32)
          asm volatile("discard.global.L2 [%0], 128;" ::"l"(tb + (size_t)ln * 128) : "memory");
      }
      s[0] = xi.zero ? s[0] : 4.0 * s[0];  // the pairing scales: 4 and 4^q, 1 for x = 0
#pragma unroll
      for (int q = 0; q < NQ; ++q) s[1 + q] *= q_scale<QS>(q, xi.zero != 0, a.qp);
      if constexpr (LANE_ACC) {
        // per-lane double-double sums, reduced across the warp once per stage below
#pragma unroll
        for (int q = 0; q <= NQ; ++q) dd_add(acc[q], s[q]);
      } else {
#pragma unroll
        for (int q = 0; q <= NQ; ++q) dd_add(acc[q], warp_sum(s[q]));
      }
    }
  }
  if (LANE_ACC && n2 > 0) {
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
  if (lane == 0 && n2 > 0) {
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
#ifdef HM_TMEM_EXCHANGE
  tmem_cta_free(tmem_base, TmemCols<T>::value);
#endif
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
