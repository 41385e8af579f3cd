// sweep_queue.cuh -- persistent work-queue sweep of the exact-SRE transforms: many states
// of different qubit counts (or one state) in one launch.
//
// The launch is one grid of resident warps that claim work units from a queue in device
// memory (an atomic counter) until it is empty.  The host lays the queue out in cost
// order: the two-pass states (12 <= n <= 21) first, largest first, then the states that
// fit one warp (n <= 11).  A unit is one warp's piece of work:
//   fused   one warp transforms and reduces XPW = 2^(11 - n) consecutive X-strings of an
//           n <= 11 state (the k_sre_fused unit with the size as a run-time value);
//   pass 1  gather + build one 1024-point row of one X-string, its 10 low butterfly
//           levels, written to a ring slot through tensor stores;
//   pass 2  one 1024-element tile of one X-string's intermediate (2^(n-11) rows x C
//           positions): the n - 11 remaining levels and the moment sums.
// A two-pass state is cut into batches of X X-strings whose intermediates fill one ring
// slot; with a lead of L batches the queue holds P1(0) .. P1(L-1), then P1(b+L) P2(b) for
// b = 0, 1, ..., then the last L P2s, so a batch's pass 2 is claimed about L batches after
// its pass 1.
// The batches of all states share one global numbering q and the ring's K slots (slot q
// mod K).  Two counters per batch replace the kernel boundaries of the stage kernels:
//   done1[q] counts finished pass-1 units: a pass-2 unit of batch q waits until it
//            reaches the batch's unit count;
//   done2[q] counts finished pass-2 units: the first pass-1 unit to reuse the slot (batch
//            q + K) waits until it reaches batch q's unit count (bunits[q]: batch q may
//            belong to an earlier, larger state than batch q + K).
// Every wait is on units that sit earlier in the queue, so they were claimed by running
// warps that never wait on later units: the sweep cannot deadlock.  Each wait still
// gives up after a bounded number of polls, records it in `err` and carries on (the host
// then reports HM_ERR_TIMEOUT), so a fault in this protocol cannot hang the GPU.
// A warp announces a finished pass-1 unit only after its tensor stores have completed;
// it does so lazily (before its next tensor store, before any wait, at exit) so that
// the store's round trip overlaps the next unit.
//
// Sums: each lane keeps double-double accumulators for the state it is working on and
// the warp adds them into its own slot of that state when it moves to another state or
// exits; a fold kernel adds every warp's slot of a state in warp order.  The order in
// which units reach a warp varies between runs, but every sum after the per-unit lane
// sums is double-double (about 1e-30 relative), so the rounded results do not depend on
// it in practice.
//
// X-strings below 2^10 have their highest set bit j inside a row.  Instead of reading a
// copy of psi with bits j and n-1 exchanged, pass 1 applies that relabelling while it
// gathers: element e of row rho reads row rho + 2^(n-11) when bit j of e is set, at
// position e with bit j cleared, and its partner at that position XOR x (the relabelled
// string x ^ 2^j ^ 2^(n-1) pairs the two halves of the top bit).  x = 0 pairs the top
// bit as well: f = (|a|^2 + |b|^2, |a|^2 - |b|^2) of the rows rho and rho + 2^(n-11).
// The FP32 kernel forms f in FP32 from an FP32 copy of psi (two roundings of order 2^-24
// per product) and never sees x = 0, which the host runs in an FP64 launch.
#pragma once
#include <cuda.h>

#include "sre_engine.cuh"
#include "sre_kernels.cuh"

namespace hm {

constexpr int QWARPS = 4;       // warps per CTA of the queue sweep
constexpr int QMAX_TMAPS = 10;  // two-pass sizes n = 12 .. 21
constexpr int QWAIT_POLLS = 1 << 22;  // default polls of a batch counter before a wait gives up (~0.3 s)

// one state of the queue
struct QState {
  const double2 *psi;   // FP64 state (one-warp units; two-pass units of the FP64 kernel)
  const float2 *psi32;  // FP32 copy (two-pass units of the FP32 kernel)
  uint64_t k_begin, k_end;  // Gray range
  long long u0, u1;         // queue units [u0, u1)
  int n;
  int X;       // two-pass: X-strings per batch (a power of two); fused: X-strings per unit
  int lgX;     // log2 X
  int nbatch;  // two-pass batches
  int q0;      // two-pass: global index of batch 0
};

struct QArgs {
  CUtensorMap tmap[QMAX_TMAPS];  // ring views per two-pass n (index n - 12)
  TmaGeom geom[QMAX_TMAPS];
  int xcap[QMAX_TMAPS];  // X-string positions per slot for that n (slot_elems / 2^(n-1))
  int tma[QMAX_TMAPS];   // 1: pass 1 stores through the tensor map; 0: plain stores
  const QState *st;
  void *ring;
  unsigned *done1, *done2;  // per global batch
  const unsigned *bunits;    // per global batch: its pass-1 (= pass-2) unit count
  unsigned long long *next;  // queue head
  double *slots;             // [nwarps][nstates][2 (1 + NQ)]
  int *err;                  // 1 after a wait gave up
  long long total;           // queue units
  long long slot_elems;      // complex elements per ring slot
  QParams qp;
  int nstates;
  int K;      // ring slots
  int chunk;  // units claimed per atomic
  int poll_limit;  // polls of a batch counter before a wait gives up
  int lead;        // batches between a batch's pass 1 and its pass 2 in the queue (>= 1)
  int stall_test;  // 1: pass-2 units of batch 0 wait for one unit more than exist (test of the bounded waits)
};

// register-bit butterflies over bits [lo, hi) of the register index, bounds at run time
// (the five stage bodies are unrolled; a warp-uniform test selects them)
template <int R, typename V>
__device__ __forceinline__ void reg_wht_rt(V (&v)[R], int lo, int hi) {
#pragma unroll
  for (int s = 0; s < ilog2c(R); ++s) {
    if (s < lo || s >= hi) continue;
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

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// lane 0 polls until *p >= target (bounded); the warp then proceeds together.  A wait
// also gives up as soon as another wait of the launch has given up (every 64 polls it
// looks at the error word), so a failed launch ends after one poll limit, not one per
// waiting unit.
__device__ __forceinline__ void warp_wait_count(const unsigned *p, unsigned target, int *err, int lane, int limit) {
  if (lane == 0) {
    int polls = 0;
    while (ld_acquire(p) < target) {
      if (++polls >= limit || ((polls & 63) == 0 && *(volatile int *)err)) {
        atomicExch(err, 1);
        break;
      }
      __nanosleep(64);
    }
  }
  __syncwarp();
}

__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// counter += v with release semantics: this thread's earlier memory operations are visible
// to whoever observes the new count with an acquire load (no separate full fence)
__device__ __forceinline__ void red_release_add(unsigned *p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T> struct QOcc { static constexpr int value = sizeof(T) == 8 ? 2 : 3; };

template <typename T, int QS>
__global__ void __launch_bounds__(QWARPS * 32, QOcc<T>::value) k_sre_queue(const __grid_constant__ QArgs a) {
  using V = typename VT<T>::V;
  constexpr int R = 32, PB = 10, NQ = QSet<QS>::NQ;
  extern __shared__ __align__(1024) unsigned char smem_q[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *sm = reinterpret_cast<V *>(smem_q) + warp * (32 * R);
  const int gwarp = blockIdx.x * QWARPS + warp;
#ifdef HM_TMEM_EXCHANGE
  // TMEM for the two-pass units' lane <-> register exchanges
  __shared__ uint32_t tmem_slot;
  const uint32_t tmem_base = tmem_cta_alloc(&tmem_slot, TmemCols<T>::value);
  const uint32_t ta = tmem_warp_addr(tmem_base);
#endif
  dd acc[NQ + 1];
#pragma unroll
  for (int t = 0; t <= NQ; ++t) acc[t] = dd{0.0, 0.0};
  bool dirty = false;
  int si = 0;
  int pending = -1;  // batch whose pass-1 unit this warp finished but has not announced
  // the warp's last tensor stores may still be reading its shared buffer: the next unit
  // waits for them right before its first shared-memory access, so that the read overlaps
  // that unit's global loads and first butterflies
  bool sm_busy = false;
  auto ready = [&]() {
    if (sm_busy) {
      if (lane == 0) bulk_wait_read_all();
      __syncwarp();
      sm_busy = false;
    }
  };
  long long u = 0, uend = 0;

  // announce the pending pass-1 unit once its tensor stores have completed (lane 0)
  auto announce = [&]() {
    if (lane == 0 && pending >= 0) {
      bulk_wait_all();
      fence_proxy_async_global();
      red_release_add(a.done1 + pending, 1u);
    }
    pending = -1;
  };
  // add the lanes' sums into this warp's slot of state si (fixed butterfly order)
  auto flush = [&]() {
#pragma unroll
    for (int t = 0; t <= NQ; ++t) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        dd other;
        other.hi = __shfl_xor_sync(0xffffffffu, acc[t].hi, o);
        other.lo = __shfl_xor_sync(0xffffffffu, acc[t].lo, o);
        dd_add_dd(acc[t], other);
      }
    }
    if (lane == 0) {
      double *sl = a.slots + ((size_t)gwarp * a.nstates + si) * 2 * (NQ + 1);
#pragma unroll
      for (int t = 0; t <= NQ; ++t) {
        dd v{sl[2 * t], sl[2 * t + 1]};
        dd_add_dd(v, acc[t]);
        sl[2 * t] = v.hi;
        sl[2 * t + 1] = v.lo;
      }
    }
#pragma unroll
    for (int t = 0; t <= NQ; ++t) acc[t] = dd{0.0, 0.0};
    dirty = false;
  };

  // Lane 0 keeps the next claim in flight: the atomic is issued one chunk ahead and its
  // result is read only when the current chunk is done, so its round trip overlaps the
  // work.  (A claimed chunk is always later than its holder's current unit, so holding it
  // cannot block the earliest unfinished unit.)
  unsigned long long claim = 0;
  if (lane == 0) claim = atomicAdd(a.next, (unsigned long long)a.chunk);
  for (;;) {
    if (u >= uend) {
      unsigned long long c0 = __shfl_sync(0xffffffffu, claim, 0);
      u = (long long)c0;
      uend = u + a.chunk < a.total ? u + a.chunk : a.total;
      if (u >= a.total) break;
      if (lane == 0) claim = atomicAdd(a.next, (unsigned long long)a.chunk);
    }
    while (a.st[si].u1 <= u) {
      if (dirty) flush();
      ++si;
    }
    const QState s = a.st[si];
    const long long p = u - s.u0;
    ++u;
    const int n = s.n;
    if (n <= 11) {
      // ---------------------------------------------------------------- fused unit
      const int NB = n - 1;
      const uint64_t kbase = s.k_begin + (uint64_t)p * (uint64_t)s.X;
      const bool lane_uniform = NB >= 5;
      V v[R];
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const uint32_t e = (uint32_t)(i * 32 + lane);
        const uint64_t xl = e >> NB, rp = e & ((1u << NB) - 1u);
        const uint64_t k = kbase + xl;
        double2 f = make_double2(0.0, 0.0);
        if (k < s.k_end) {
          const uint64_t x = gray_code(k);
          if (x == 0) {
            f = zero_pair(ld_psi(s.psi + rp), ld_psi(s.psi + rp + (1ull << NB)));
          } else {
            const int j = 63 - __clzll((long long)x);
            const uint64_t r = insert0(rp, j);
            f = conj_mul(ld_psi(s.psi + r), ld_psi(s.psi + (r ^ x)));
            if (!lane_uniform) {
              f.x += f.x;
              f.y += f.y;
            }
          }
        }
        v[i].x = (T)f.x;
        v[i].y = (T)f.y;
      }
      reg_wht_rt<R>(v, 0, NB - 5);
      ready();
      transpose_ab<R>(v, sm, lane);
      reg_wht_rt<R>(v, 0, NB < 5 ? NB : 5);
      double sums[NQ + 1];
      lane_moments<R, QS>(v, sums, a.qp, sm, lane);
      if (lane_uniform) {
        const uint64_t k = kbase + (((uint64_t)lane * R) >> NB);
        const bool act = k < s.k_end;
        const bool xz = gray_code(k) == 0;
        sums[0] = act ? (xz ? sums[0] : 4.0 * sums[0]) : 0.0;
#pragma unroll
        for (int t = 0; t < NQ; ++t) sums[1 + t] = act ? sums[1 + t] * q_scale<QS>(t, xz, a.qp) : 0.0;
      }
#pragma unroll
      for (int t = 0; t <= NQ; ++t) dd_add(acc[t], sums[t]);
      dirty = true;
      continue;
    }
    // ------------------------------------------------------------------ two-pass unit
    const int hi = n - 11;  // row bits of an X-string's intermediate
    const int lgU = s.lgX + hi;
    const long long U = 1ll << lgU;  // units per pass per batch
    // segments s = 0 .. nbatch + lead - 1 hold P1(s) (s < nbatch) then P2(s - lead)
    // (s >= lead): zone A = P1 only, zone B = both, zone C = P2 only
    int b, pass;
    long long r;
    {
      const int L = a.lead, nb = s.nbatch;
      const int za = L < nb ? L : nb;
      const long long A = (long long)za << lgU;
      const long long B = (long long)(nb > L ? nb - L : 0) << (lgU + 1);
      if (p < A) {
        b = (int)(p >> lgU), pass = 1, r = p & (U - 1);
      } else if (p < A + B) {
        const long long p2 = p - A;
        const int sg = L + (int)(p2 >> (lgU + 1));
        const long long w = p2 & (2 * U - 1);
        pass = w < U ? 1 : 2;
        b = w < U ? sg : sg - L;
        r = w & (U - 1);
      } else {
        const long long p3 = p - A - B;
        const int sg = (L > nb ? L : nb) + (int)(p3 >> lgU);
        b = sg - L, pass = 2, r = p3 & (U - 1);
      }
    }
    const int q = s.q0 + b;
    const int slot = q % a.K;
    const int xs = (int)(r & (s.X - 1));
    const uint64_t sub = (uint64_t)(r >> s.lgX);
    const uint64_t k = s.k_begin + (uint64_t)b * s.X + xs;
    const bool active = k < s.k_end;
    const int ti = n - 12;
    const int xcap = a.xcap[ti];
    V *inter_x = reinterpret_cast<V *>(a.ring) + (size_t)slot * a.slot_elems + ((size_t)xs << (n - 1));
    if (pass == 1) {
      if (q >= a.K) {
        announce();
        // batch q - K may belong to an earlier state, with its own unit count
        warp_wait_count(a.done2 + (q - a.K), a.bunits[q - a.K], a.err, lane, a.poll_limit);
        if (lane == 0) fence_proxy_async_global();  // the slot's reads come before the new stores
      }
      if (active) {
        const uint64_t x = gray_code(k);
        const uint64_t H = 1ull << hi;
        // the FP64 kernel gathers the FP64 state; the FP32 kernel its FP32 copy (x = 0 never
        // reaches it: the host runs every x = 0 transform in FP64)
        using VS = typename VT<T>::V;
        const VS *ps = sizeof(T) == 8 ? reinterpret_cast<const VS *>(s.psi) : reinterpret_cast<const VS *>(s.psi32);
        V v[R];
        if (x >= (1ull << PB)) {
          const int jt = 63 - __clzll((long long)x);
          const uint64_t rH = insert0(sub, jt - PB);
          const uint64_t sH = rH ^ (x >> PB);
          const uint32_t xL = (uint32_t)(x & ((1ull << PB) - 1ull));
          const VS *rowA = ps + (rH << PB), *rowB = ps + (sH << PB);
#pragma unroll
          for (int i = 0; i < R; ++i) {
            const uint32_t e = (uint32_t)(i * 32 + lane);
            v[i] = conj_mul(ld_psi(rowA + e), ld_psi(rowB + (e ^ xL)));
          }
        } else if (x != 0) {
          const int j = 63 - __clzll((long long)x);
          const uint32_t xl = (uint32_t)x, jm = 1u << j;
          const VS *row0 = ps + (sub << PB), *row1 = ps + ((sub + H) << PB);
#pragma unroll
          for (int i = 0; i < R; ++i) {
            const uint32_t e = (uint32_t)(i * 32 + lane);
            const VS *row = (e & jm) ? row1 : row0;
            const uint32_t eh = e & ~jm;
            v[i] = conj_mul(ld_psi(row + eh), ld_psi(row + (eh ^ xl)));
          }
        } else if constexpr (sizeof(T) == 8) {
          const double2 *row0 = s.psi + (sub << PB), *row1 = s.psi + ((sub + H) << PB);
#pragma unroll
          for (int i = 0; i < R; ++i) {
            const uint32_t e = (uint32_t)(i * 32 + lane);
            const double2 f = zero_pair(ld_psi(row0 + e), ld_psi(row1 + e));
            v[i].x = (T)f.x;
            v[i].y = (T)f.y;
          }
        }
        reg_wht<R, 0, 5>(v);
        ready();
#ifdef HM_TMEM_EXCHANGE
        tmem_row(v, ta);
#else
        transpose_ab<R>(v, sm, lane);
#endif
        reg_wht<R, 0, 5>(v);
        if (a.tma[ti]) {
#pragma unroll
          for (int i = 0; i < R; ++i) sm[i * 32 + lane] = v[i];
          fence_proxy_async_smem();
          __syncwarp();
          announce();  // the previous unit's stores completed long ago in most cases
          if (lane == 0) {
            const TmaGeom g = a.geom[ti];
            const int xcoord = slot * xcap + xs;
            for (int b2 = 0; b2 < g.nb2; ++b2)
              for (int b0 = 0; b0 < g.nb0; ++b0)
                tma_store_4d(&a.tmap[ti], sm + (size_t)b2 * g.box2 * g.C + (size_t)b0 * (g.box0 / 2), b0 * g.box0,
                             (int)sub, b2 * g.box2, xcoord);
            bulk_commit();
          }
          sm_busy = true;
          pending = q;
        } else {
          // tile rows too narrow for a tensor map (FP32 at n = 21: 8 bytes): plain stores of
          // position p = 32 i + lane to tile p >> LOGC, column p mod C
          const int LOGC = PB - hi;
#pragma unroll
          for (int i = 0; i < R; ++i) {
            const uint32_t pp = (uint32_t)(i * 32 + lane);
            const uint32_t t = pp >> LOGC, cc = pp & ((1u << LOGC) - 1u);
            __stcg(inter_x + (((size_t)t << (hi + LOGC)) + (sub << LOGC) + cc), v[i]);
          }
          __threadfence();
          __syncwarp();
          announce();
          if (lane == 0) atomicAdd(a.done1 + q, 1u);
        }
      } else {
        announce();
        if (lane == 0) red_release_add(a.done1 + q, 1u);
      }
    } else {
      announce();
      warp_wait_count(a.done1 + q, (unsigned)U + (a.stall_test && q == 0 ? 1u : 0u), a.err, lane, a.poll_limit);
      if (active) {
        const int LOGC = PB - hi;
        const V *tile = inter_x + (sub << PB);
        V v[R];
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = __ldcg(tile + i * 32 + lane);
        if (LOGC >= 5) {
          reg_wht_rt<R>(v, LOGC - 5, 5);
        } else {
          reg_wht<R, 0, 5>(v);
          ready();
#ifdef HM_TMEM_EXCHANGE
          switch (hi) {  // warp-uniform
            case 6: tmem_tile<6>(v, ta); break;
            case 7: tmem_tile<7>(v, ta); break;
            case 8: tmem_tile<8>(v, ta); break;
            case 9: tmem_tile<9>(v, ta); break;
            default: tmem_tile<10>(v, ta); break;
          }
          reg_wht_rt<R>(v, 0, 5 - LOGC);
#else
          transpose_ab<R>(v, sm, lane);
          reg_wht_rt<R>(v, LOGC, 5);
#endif
        }
        double sums[NQ + 1];
        ready();  // the generic-q moments stage the values in the shared buffer
        lane_moments<R, QS>(v, sums, a.qp, sm, lane);
        const bool xz = gray_code(k) == 0;
        dd_add(acc[0], xz ? sums[0] : 4.0 * sums[0]);
#pragma unroll
        for (int t = 0; t < NQ; ++t) dd_add(acc[1 + t], sums[1 + t] * q_scale<QS>(t, xz, a.qp));
        dirty = true;
      }
      __syncwarp();
      if (lane == 0) red_release_add(a.done2 + q, 1u);
    }
  }
  announce();
  if (dirty) flush();
  if (lane == 0) bulk_wait_all();
#ifdef HM_TMEM_EXCHANGE
  tmem_cta_free(tmem_base, TmemCols<T>::value);
#endif
}

// fold of every warp's slot of each state, in warp order: out[s][2t], out[s][2t + 1]
__global__ void k_queue_fold(const double *__restrict__ slots, int nwarps, int nstates, int nsum, double *out);

}  // namespace hm
