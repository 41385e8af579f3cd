// adjoint.cu -- value and gradient of the exact SRE_q with respect to Re psi and Im psi.
//
// No reference counterpart.  Forward, per X-string x (the complex pairing of the SRE
// engine): W = WHT_{n-1}(f), f(r') = conj a b with a = psi(r), b = psi(r ^ x), r in
// V0(x); F = 2 Re W, 2 Im W and m = sum_x sum (F^2)^q.  Then
//     Gamma = WHT_{n-1}( c_q (Re W^{2q-1} + i Im W^{2q-1}) ),  c_q = 2q 4^q,
// is dm/dRe f + i dm/dIm f, and with f = conj(a) b
//     dm/da = conj(Gamma) b,   dm/db = Gamma a     (complex gradient d/dRe + i d/dIm).
// For x = 0 (h = (|a|^2 + |b|^2, |a|^2 - |b|^2), b = psi(r' + 2^(n-1)), F = Re W, Im W):
//     dm/da = 2 (Gamma_re + Gamma_im) a,   dm/db = 2 (Gamma_re - Gamma_im) b,   c_q = 2q.
// Writing either case as G_x(u) psi(u ^ x) (G_x(u) = conj Gamma for u = r, Gamma for
// u = r ^ x; 2 (Gamma_re +- Gamma_im) for x = 0), the gradient is
//     dm/dpsi(u) = sum_x G_x(u) psi(u ^ x).
// The forward transforms are recomputed per x; G is produced for a chunk of X-strings at
// a time and folded into the gradient by one thread per u (no atomics).  Finally
// dSRE = -dm / (m ln 2).
#include <math.h>

#include "hm_ctx.h"
#include "sre_launch.cuh"

namespace hm {

namespace {

constexpr int R = 32, PB = 10;

struct AdjArgs {
  const double2 *psi;
  const double2 *psi_sw[16];
  double2 *ring;     // chunk x 2^(n-1)   (two-pass intermediate)
  double2 *G;        // chunk x 2^n
  double2 *grad;     // 2^n, accumulated dm/dpsi
  double *mpart;     // per warp: sum (F^2)^q (plain), folded at the end
  double q, cq_x, cq_0;
  int n, U, chunk;
  uint64_t x0;  // first X-string (natural order) of the chunk
  int nx;
};

// y^e for an integer 0 <= e <= 7: binary powering in three branch-free steps, so that
// the unrolled register sweep keeps its instruction-level parallelism
__device__ __forceinline__ double powi7(double y, int e) {
  double r = 1.0, b = y;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    r = (e & 1) ? r * b : r;
    b *= b;
    e >>= 1;
  }
  return r;
}

// pointwise map on every register: accumulate sum (W^2)^q, replace W by c W^{2q-1}.
// Q = 2, 3: compile-time exponent, unrolled over the registers; Q = 0: q at run time
// (1 <= q <= 8), in a rolled loop over the lane's own slots of the warp's shared buffer
// (an unrolled sweep of the run-time power spills registers).
template <int Q>
__device__ __forceinline__ double adj_pointwise(double2 (&v)[R], int q, double cq, double2 *sm, int lane) {
  if constexpr (Q == 0) {
#pragma unroll
    for (int i = 0; i < R; ++i) sm[lane + 32 * i] = v[i];
    double m = 0.0;
#pragma unroll 1
    for (int i = 0; i < R; ++i) {
      double2 w = sm[lane + 32 * i];
      const double a2 = w.x * w.x, b2 = w.y * w.y;
      const double pa = powi7(a2, q - 1), pb = powi7(b2, q - 1);
      m += pa * a2 + pb * b2;
      w.x = cq * w.x * pa;
      w.y = cq * w.y * pb;
      sm[lane + 32 * i] = w;
    }
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = sm[lane + 32 * i];
    __syncwarp();  // the buffer is rewritten by the next transpose
    return m;
  } else {
    double m0 = 0.0, m1 = 0.0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const double a = v[i].x, b = v[i].y;
      const double a2 = a * a, b2 = b * b;
      const double pa = Q == 2 ? a2 : a2 * a2, pb = Q == 2 ? b2 : b2 * b2;  // (W^2)^(q-1)
      m0 += pa * a2;
      m1 += pb * b2;
      v[i].x = cq * a * pa;
      v[i].y = cq * b * pb;
    }
    return m0 + m1;
  }
}

// layout B -> layout A (inverse of transpose_ab)
__device__ __forceinline__ void transpose_ba(double2 (&v)[R], double2 *sm, int lane) {
  constexpr int LOGR = 5, SW = 7;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int e = lane * R + i;
    sm[e ^ ((e >> LOGR) & SW)] = v[i];
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int e = i * 32 + lane;
    v[i] = sm[e ^ ((e >> LOGR) & SW)];
  }
  __syncwarp();
}

// write G for the pair (u1 = row A element, u2 = row B element) of one x
__device__ __forceinline__ void put_G(double2 *Gx, uint64_t u1, uint64_t u2, double2 gam, bool xzero) {
  if (xzero) {
    Gx[u1] = make_double2(2.0 * (gam.x + gam.y), 0.0);
    Gx[u2] = make_double2(2.0 * (gam.x - gam.y), 0.0);
  } else {
    Gx[u1] = make_double2(gam.x, -gam.y);
    Gx[u2] = gam;
  }
}

// ---------------------------------------------------------------------------------
// n <= 11: one warp per X-string does everything
template <int NB>
__global__ void __launch_bounds__(128) k_adj_fused(AdjArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  const int xi = blockIdx.x * 4 + warp;
  double mloc = 0.0;
  if (xi < a.nx) {
    const uint64_t x = a.x0 + xi;
    const bool xz = (x == 0);
    const int j = xz ? NB : 63 - __clzll((long long)x);
    double2 v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint32_t e = (uint32_t)(i * 32 + lane);
      double2 f = make_double2(0.0, 0.0);
      if (e < (1u << NB)) {
        if (xz)
          f = zero_pair(a.psi[e], a.psi[e + (1u << NB)]);
        else {
          const uint64_t r = insert0(e, j);
          f = conj_mul(a.psi[r], a.psi[r ^ x]);
        }
      }
      v[i] = f;
    }
    if constexpr (NB > 5) reg_wht<R, 0, NB - 5>(v);
    transpose_ab<R>(v, sm, lane);
    reg_wht<R, 0, (NB < 5 ? NB : 5)>(v);
    const int qi = (int)a.q;
    mloc = adj_pointwise<0>(v, qi, xz ? a.cq_0 : a.cq_x, sm, lane) * (xz ? 1.0 : pow_q_dev(4.0, a.q));
    reg_wht<R, 0, (NB < 5 ? NB : 5)>(v);
    transpose_ba(v, sm, lane);
    if constexpr (NB > 5) reg_wht<R, 0, NB - 5>(v);
    double2 *Gx = a.G + (size_t)xi * ((size_t)1 << a.n);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint32_t e = (uint32_t)(i * 32 + lane);
      if (e < (1u << NB)) {
        const uint64_t u1 = xz ? e : insert0(e, j);
        const uint64_t u2 = xz ? e + (1u << NB) : (u1 ^ x);
        put_G(Gx, u1, u2, v[i], xz);
      }
    }
  }
  mloc = warp_sum(mloc);
  if (lane == 0) a.mpart[blockIdx.x * 4 + warp] += mloc;
}

// ---------------------------------------------------------------------------------
// n >= 12.  Pass 1 (forward, low bits) for (x, row); x = 0 uses the zero-pair build.
template <int HI>
__global__ void __launch_bounds__(128) k_adj_p1(AdjArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  const long long u = (long long)blockIdx.x * 4 + warp;
  if (u >= (long long)a.nx * a.U) return;
  const int xi = (int)(u / a.U);
  const uint64_t rho = (uint64_t)(u % a.U);
  const uint64_t x = a.x0 + xi;
  double2 *ring = a.ring + (size_t)xi * ((size_t)1 << (a.n - 1));
  if (x == 0) {
    // pairing on the top bit: rows rho and rho + 2^(n-1-PB)
    constexpr int LOGC = PB - HI;
    double2 v[R];
    const double2 *rowA = a.psi + (rho << PB), *rowB = a.psi + ((rho + (1ull << (a.n - 1 - PB))) << PB);
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = zero_pair(rowA[i * 32 + lane], rowB[i * 32 + lane]);
    reg_wht<R, 0, 5>(v);
    transpose_ab<R>(v, sm, lane);
    reg_wht<R, 0, 5>(v);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint32_t p = (uint32_t)(i * 32 + lane);
      const uint32_t t = p >> LOGC, c = p & ((1u << LOGC) - 1u);
      ring[((size_t)t << (HI + LOGC)) + (rho << LOGC) + c] = v[i];
    }
    return;
  }
  XInfo xi_;
  xi_.active = 1;
  xi_.sw = -1;
  xi_.xt = x;
  xi_.jt = 63 - __clzll((long long)x);
  if (xi_.jt < PB) {
    xi_.sw = xi_.jt;
    xi_.xt = (x ^ (1ull << xi_.jt)) | (1ull << (a.n - 1));
    xi_.jt = a.n - 1;
  }
  const double2 *src = xi_.sw < 0 ? a.psi : a.psi_sw[xi_.sw];
  p1_unit<R, HI, false>(src, xi_, rho, ring, sm, lane);
}

// Pass 2: forward high bits, pointwise map, backward high bits, in place
template <int HI>
__global__ void __launch_bounds__(128) k_adj_p2(AdjArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  const long long u = (long long)blockIdx.x * 4 + warp;
  double mloc = 0.0;
  if (u < (long long)a.nx * a.U) {
    constexpr int LOGC = PB - HI;
    const int xi = (int)(u / a.U);
    const uint64_t tile = (uint64_t)(u % a.U);
    const bool xz = (a.x0 + xi == 0);
    double2 *tp = a.ring + (size_t)xi * ((size_t)1 << (a.n - 1)) + (tile << PB);
    double2 v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = tp[i * 32 + lane];
    if constexpr (LOGC >= 5) {
      reg_wht<R, LOGC - 5, 5>(v);
    } else {
      reg_wht<R, 0, 5>(v);
      transpose_ab<R>(v, sm, lane);
      reg_wht<R, LOGC, 5>(v);
    }
    mloc = adj_pointwise<0>(v, (int)a.q, xz ? a.cq_0 : a.cq_x, sm, lane) * (xz ? 1.0 : pow_q_dev(4.0, a.q));
    if constexpr (LOGC >= 5) {
      reg_wht<R, LOGC - 5, 5>(v);
    } else {
      reg_wht<R, LOGC, 5>(v);
      transpose_ba(v, sm, lane);
      reg_wht<R, 0, 5>(v);
    }
#pragma unroll
    for (int i = 0; i < R; ++i) tp[i * 32 + lane] = v[i];
  }
  mloc = warp_sum(mloc);
  if (lane == 0) a.mpart[blockIdx.x * 4 + warp] += mloc;
}

// Pass 1 backward (low bits) for (x, row): Gamma of the row -> G_x at both partners
template <int HI>
__global__ void __launch_bounds__(128) k_adj_p1b(AdjArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  const long long u = (long long)blockIdx.x * 4 + warp;
  if (u >= (long long)a.nx * a.U) return;
  constexpr int LOGC = PB - HI;
  const int xi = (int)(u / a.U);
  const uint64_t rho = (uint64_t)(u % a.U);
  const uint64_t x = a.x0 + xi;
  const double2 *ring = a.ring + (size_t)xi * ((size_t)1 << (a.n - 1));
  double2 v[R];
  // position p = 32 i + l of the row holds element k = R l + i: loading it into
  // register i of lane l gives layout B
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const uint32_t p = (uint32_t)(i * 32 + lane);
    const uint32_t t = p >> LOGC, c = p & ((1u << LOGC) - 1u);
    v[i] = ring[((size_t)t << (HI + LOGC)) + (rho << LOGC) + c];
  }
  reg_wht<R, 0, 5>(v);
  transpose_ba(v, sm, lane);
  reg_wht<R, 0, 5>(v);  // now layout A: register i of lane l holds element e = 32 i + l
  double2 *Gx = a.G + (size_t)xi * ((size_t)1 << a.n);
  if (x == 0) {
    const uint64_t top = 1ull << (a.n - 1);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint64_t u1 = (rho << PB) | (uint32_t)(i * 32 + lane);
      put_G(Gx, u1, u1 + top, v[i], true);
    }
    return;
  }
  uint64_t xt = x;
  int jt = 63 - __clzll((long long)x), sw = -1;
  if (jt < PB) {
    sw = jt;
    xt = (x ^ (1ull << jt)) | (1ull << (a.n - 1));
    jt = a.n - 1;
  }
  const uint64_t rH = insert0(rho, jt - PB), sH = rH ^ (xt >> PB);
  const uint32_t xL = (uint32_t)(xt & ((1ull << PB) - 1ull));
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const uint32_t e = (uint32_t)(i * 32 + lane);
    uint64_t u1 = (rH << PB) | e, u2 = (sH << PB) | (e ^ xL);
    if (sw >= 0) {
      u1 = swap_bits(u1, sw, a.n - 1);
      u2 = swap_bits(u2, sw, a.n - 1);
    }
    put_G(Gx, u1, u2, v[i], false);
  }
}

// grad(u) += sum over the chunk's X-strings of G_x(u) psi(u ^ x).  A block covers 32
// consecutive u; its 8 warps take fixed eighths of the chunk's X-strings (4 interleaved
// sums each, so several loads are in flight), and warp 0 adds the eighths in order: the
// result does not depend on scheduling.
constexpr int ACC_SEGS = 8;
__global__ void __launch_bounds__(32 * ACC_SEGS) k_adj_acc(AdjArgs a) {
  __shared__ double2 part[ACC_SEGS][32];
  const uint64_t len = 1ull << a.n;
  const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5;
  const int per = (a.nx + ACC_SEGS - 1) / ACC_SEGS;
  const int xb = min(a.nx, seg * per), xe = min(a.nx, xb + per);
  for (uint64_t base = blockIdx.x * 32ull; base < len; base += (uint64_t)gridDim.x * 32ull) {
    const uint64_t uu = base + lane;
    double gr[4] = {0.0, 0.0, 0.0, 0.0}, gi[4] = {0.0, 0.0, 0.0, 0.0};
    if (uu < len) {
      int xi = xb;
      for (; xi + 3 < xe; xi += 4) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double2 g = a.G[(size_t)(xi + j) * len + uu];
          const double2 p = __ldg(a.psi + (uu ^ (a.x0 + xi + j)));
          gr[j] += g.x * p.x - g.y * p.y;
          gi[j] += g.x * p.y + g.y * p.x;
        }
      }
      for (; xi < xe; ++xi) {
        const double2 g = a.G[(size_t)xi * len + uu];
        const double2 p = __ldg(a.psi + (uu ^ (a.x0 + xi)));
        gr[0] += g.x * p.x - g.y * p.y;
        gi[0] += g.x * p.y + g.y * p.x;
      }
    }
    part[seg][lane] = make_double2((gr[0] + gr[1]) + (gr[2] + gr[3]), (gi[0] + gi[1]) + (gi[2] + gi[3]));
    __syncthreads();
    if (seg == 0 && uu < len) {
      double2 sum = part[0][lane];
#pragma unroll
      for (int k = 1; k < ACC_SEGS; ++k) {
        sum.x += part[k][lane].x;
        sum.y += part[k][lane].y;
      }
      double2 o = a.grad[uu];
      o.x += sum.x;
      o.y += sum.y;
      a.grad[uu] = o;
    }
    __syncthreads();
  }
}

__global__ void k_adj_finish(double2 *grad, uint64_t len, const double *mpart, int nw, double *m_out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < nw; i += blockDim.x) s += mpart[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double m = sh[0];
  const double scale = -1.0 / (m * 0.69314718055994530942);
  for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) {
    double2 g = grad[i];
    grad[i] = make_double2(g.x * scale, g.y * scale);
  }
  if (threadIdx.x == 0) *m_out = m;
}


// ---------------------------------------------------------------------------------
// n >= 12, X-strings x >= 2^PB: stage kernels.  Batch b holds the X consecutive
// X-strings x_begin + b X + xs (aligned, so they share their pairing bit and the rows
// rH, sH of every rho; only the low bits xs of x differ).  Stage t runs four kernels,
// one per kind of unit (independent work inside the stage):
//   k_adjs_grad  gradient units of batch t-3 (row rho, kind A/B, part of the row),
//   k_adjs_p1b   backward low of batch t-2 (Gamma rows, natural element order, into `gam`),
//   k_adjs_p2f   forward high + pointwise + backward high of batch t-1 (in place),
//   k_adjs_p1    pass 1 of batch t,
// with the ring in 3 slots and `gam` in 2.  One kernel per kind keeps each kernel's code
// small: a single kernel holding all four unrolled unit bodies stalled on instruction
// fetch for more than half of its cycles.  The kernels are chained by programmatic
// dependent launch; each one waits for its predecessor (and so, transitively, for all
// earlier kernels: every CTA waits before it exits) before its first access that
// depends on an earlier stage, and pass 1 runs its psi reads and butterflies before.
// A gradient unit owns its rows and part for the whole batch: kind A adds
// sum_xs conj(Gamma_xs(e)) psi_sH(e ^ xL) to row rH, kind B adds
// sum_xs Gamma_xs(e ^ xL) psi_rH(e ^ xL) to row sH at e.  No two units of a stage
// touch the same gradient entry and each entry's sum runs in a fixed order.
constexpr int ADJ_WARPS = 4;

struct AdjStageArgs {
  const double2 *psi;
  double2 *ring;    // 3 slots x X x 2^(n-1), tile-major (pass-1 layout)
  double2 *gam;     // 2 slots x X x 2^(n-1), Gamma rows in natural element order
  double2 *grad;    // 2^n, unscaled dm/dpsi
  double2 *gpart;   // (ng - 1) x 2^n partial gradients of X-string groups 1 .. ng-1
  double *mpart;    // per warp of k_adjs_p2f: sum of its pointwise-unit moments
  unsigned *stage;  // [0] stage index of node 0 of the current graph replay
  uint64_t x_begin;
  double cq, q4;    // c_q and 4^q for x != 0
  int q, n, X, nbatch;
  int ng;           // X-string groups per gradient unit row (power of two, divides X)
  int node;         // stage offset of this launch in the captured graph
};

__device__ __forceinline__ long long adj_stage_index(const AdjStageArgs &a) {
  // the base changes only between graph replays, after every node of a replay finished
  return (long long)*(volatile unsigned *)a.stage + a.node;
}

// Gradient unit: destination elements p = 32 i + lane, i in [part * GR, +GR), of row rH
// (kind 0) or row sH (kind 1) of batch b, for the X-strings of group xg (X / ng
// consecutive ones; group 0 adds into the gradient, group g > 0 into partial buffer
// g - 1, folded in at the end in group order).  Every X-string of the group adds
//   kind 0:  conj(Gamma_x(p)) psi(sH, p ^ xL)       (grad at u1 = rH p)
//   kind 1:  Gamma_x(p ^ xL)  psi(rH, p ^ xL)       (grad at u2 = sH p)
// gathered at permuted addresses (no shuffles), GX X-strings' loads in flight at once,
// summed in the order of xs.
constexpr int GR = 1, GX = 8;
constexpr int GPARTS = R / GR;  // units per row and kind

__device__ __forceinline__ void adj_grad_unit(const AdjStageArgs &a, long long b, uint64_t rho, int kind, int part,
                                              int xg, int lane) {
  const uint64_t xlen = 1ull << (a.n - 1);
  const uint64_t xb = a.x_begin + (uint64_t)b * a.X;  // aligned to X: xs occupies the low bits
  const int jt = 63 - __clzll((long long)xb);
  const uint64_t rH = insert0(rho, jt - PB), sH = rH ^ (xb >> PB);
  const uint32_t xLb = (uint32_t)(xb & ((1u << PB) - 1u));
  const double2 *gam_b = a.gam + (size_t)(b & 1) * a.X * xlen + (rho << PB);
  const double2 *rowA = a.psi + (rH << PB), *rowB = a.psi + (sH << PB);
  double2 acc[GR];
#pragma unroll
  for (int j = 0; j < GR; ++j) acc[j] = make_double2(0.0, 0.0);
  const int xpg = a.X / a.ng, xs_end = (xg + 1) * xpg;
#pragma unroll 1
  for (int xs0 = xg * xpg; xs0 < xs_end; xs0 += GX) {
    double2 g[GX][GR], w[GX][GR];
#pragma unroll
    for (int u = 0; u < GX; ++u) {
      const int xs = xs0 + u < xs_end ? xs0 + u : xs0;  // group < GX: repeat a valid one, masked below
      const double2 *g_row = gam_b + (size_t)xs * xlen;
      const uint32_t xL = xLb | (uint32_t)xs;
#pragma unroll
      for (int j = 0; j < GR; ++j) {
        const uint32_t p = (uint32_t)((part * GR + j) * 32 + lane);
        if (kind == 0) {
          g[u][j] = __ldcg(g_row + p);
          w[u][j] = __ldg(rowB + (p ^ xL));
        } else {
          g[u][j] = __ldcg(g_row + (p ^ xL));
          w[u][j] = __ldg(rowA + (p ^ xL));
        }
      }
    }
#pragma unroll
    for (int u = 0; u < GX; ++u) {
      if (xs0 + u >= xs_end) break;
#pragma unroll
      for (int j = 0; j < GR; ++j) {
        const double2 gg = g[u][j], ww = w[u][j];
        if (kind == 0) {
          acc[j].x += gg.x * ww.x + gg.y * ww.y;
          acc[j].y += gg.x * ww.y - gg.y * ww.x;
        } else {
          acc[j].x += gg.x * ww.x - gg.y * ww.y;
          acc[j].y += gg.x * ww.y + gg.y * ww.x;
        }
      }
    }
  }
  double2 *dst = xg == 0 ? a.grad : a.gpart + ((size_t)(xg - 1) << a.n);
  double2 *row = dst + ((kind == 0 ? rH : sH) << PB);
#pragma unroll
  for (int j = 0; j < GR; ++j) {
    const uint32_t p = (uint32_t)((part * GR + j) * 32 + lane);
    double2 o = row[p];
    o.x += acc[j].x;
    o.y += acc[j].y;
    row[p] = o;
  }
}

// warps per CTA and CTAs per SM of the gradient kernel (no 32R-register tiles: 16 warps
// per SM)
constexpr int GRAD_WARPS = 4, GRAD_CTAS = 4;

__global__ void __launch_bounds__(GRAD_WARPS * 32, GRAD_CTAS) k_adjs_grad(AdjStageArgs a) {
  const long long t = adj_stage_index(a);
  allow_next_grid();
  wait_prior_grid();  // reads Gamma of the previous stage, updates the gradient rows
  if (t < 3 || t - 3 >= a.nbatch) return;
  const int lane = threadIdx.x & 31;
  const int gwarp = blockIdx.x * GRAD_WARPS + (threadIdx.x >> 5), nwarps = gridDim.x * GRAD_WARPS;
  const long long nu = 2 * GPARTS * (long long)(1ull << (a.n - 1 - PB));
  for (long long u = gwarp; u < nu * a.ng; u += nwarps) {
    const long long v = u % nu;
    adj_grad_unit(a, t - 3, (uint64_t)(v / (2 * GPARTS)), (int)((v / GPARTS) & 1), (int)(v % GPARTS), (int)(u / nu),
                  lane);
  }
}

// grad += gpart[0] + gpart[1] + ... (in group order)
__global__ void k_adj_fold_groups(double2 *grad, const double2 *gpart, int nparts, uint64_t len) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    double2 g = grad[i];
    for (int k = 0; k < nparts; ++k) {
      const double2 p = gpart[(size_t)k * len + i];
      g.x += p.x;
      g.y += p.y;
    }
    grad[i] = g;
  }
}

// backward over the low bits of one row of batch t-2; Gamma in natural element order
template <int HI>
__global__ void __launch_bounds__(ADJ_WARPS * 32, 2) k_adjs_p1b(AdjStageArgs a) {
  constexpr int LOGC = PB - HI;
  extern __shared__ __align__(16) unsigned char smraw[];
  const long long t = adj_stage_index(a);
  allow_next_grid();
  wait_prior_grid();  // reads the previous stage's forward-high rows, rewrites a Gamma slot
  if (t < 2 || t - 2 >= a.nbatch) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  const int gwarp = blockIdx.x * ADJ_WARPS + warp, nwarps = gridDim.x * ADJ_WARPS;
  const uint64_t xlen = 1ull << (a.n - 1);
  const long long per = (long long)a.X << HI, b = t - 2;
  for (long long r = gwarp; r < per; r += nwarps) {
    const int xs = (int)(r % a.X);
    const uint64_t rho = (uint64_t)(r / a.X);
    const double2 *ring_x = a.ring + ((size_t)(b % 3) * a.X + xs) * xlen;
    double2 v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const uint32_t p = (uint32_t)(i * 32 + lane);
      const uint32_t tt = p >> LOGC, cc = p & ((1u << LOGC) - 1u);
      v[i] = __ldcg(ring_x + ((size_t)tt << (HI + LOGC)) + (rho << LOGC) + cc);
    }
    reg_wht<R, 0, 5>(v);
    transpose_ba(v, sm, lane);
    reg_wht<R, 0, 5>(v);  // layout A: register i of lane l holds element 32 i + l
    double2 *g_row = a.gam + ((size_t)(b & 1) * a.X + xs) * xlen + (rho << PB);
#pragma unroll
    for (int i = 0; i < R; ++i) __stcg(g_row + i * 32 + lane, v[i]);
  }
}

// forward over the row bits, pointwise map, backward over the row bits (batch t-1, in
// place in the ring); QA = q for q = 2, 3, else 0 (q at run time)
template <int HI, int QA>
__global__ void __launch_bounds__(ADJ_WARPS * 32, 2) k_adjs_p2f(AdjStageArgs a) {
  constexpr int LOGC = PB - HI;
  extern __shared__ __align__(16) unsigned char smraw[];
  const long long t = adj_stage_index(a);
  allow_next_grid();
  wait_prior_grid();  // reads the previous stage's pass-1 rows; updates the moment slots
  if (t < 1 || t - 1 >= a.nbatch) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  const int gwarp = blockIdx.x * ADJ_WARPS + warp, nwarps = gridDim.x * ADJ_WARPS;
  const uint64_t xlen = 1ull << (a.n - 1);
  const long long per = (long long)a.X << HI, b = t - 1;
  double mloc = 0.0;
  for (long long r = gwarp; r < per; r += nwarps) {
    const int xs = (int)(r % a.X);
    const uint64_t tile = (uint64_t)(r / a.X);
    double2 *tp = a.ring + ((size_t)(b % 3) * a.X + xs) * xlen + (tile << PB);
    double2 v[R];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = __ldcg(tp + i * 32 + lane);
    if constexpr (LOGC >= 5) {
      reg_wht<R, LOGC - 5, 5>(v);
    } else {
      reg_wht<R, 0, 5>(v);
      transpose_ab<R>(v, sm, lane);
      reg_wht<R, LOGC, 5>(v);
    }
    mloc += adj_pointwise<QA>(v, a.q, a.cq, sm, lane) * a.q4;
    if constexpr (LOGC >= 5) {
      reg_wht<R, LOGC - 5, 5>(v);
    } else {
      reg_wht<R, LOGC, 5>(v);
      transpose_ba(v, sm, lane);
      reg_wht<R, 0, 5>(v);
    }
#pragma unroll
    for (int i = 0; i < R; ++i) __stcg(tp + i * 32 + lane, v[i]);
  }
  mloc = warp_sum(mloc);
  if (lane == 0) a.mpart[gwarp] += mloc;
}

// pass 1 (forward over the low bits) of batch t
template <int HI>
__global__ void __launch_bounds__(ADJ_WARPS * 32, 2) k_adjs_p1(AdjStageArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const long long t = adj_stage_index(a);
  allow_next_grid();
  if (t >= a.nbatch) {
    wait_prior_grid();
    return;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  const int gwarp = blockIdx.x * ADJ_WARPS + warp, nwarps = gridDim.x * ADJ_WARPS;
  const uint64_t xlen = 1ull << (a.n - 1);
  const long long per = (long long)a.X << HI;
  // the slot is the one that the previous stage's backward-low units read
  auto pre = [] { wait_prior_grid(); };
  for (long long r = gwarp; r < per; r += nwarps) {
    const int xs = (int)(r % a.X);
    const uint64_t rho = (uint64_t)(r / a.X);
    const uint64_t x = a.x_begin + (uint64_t)t * a.X + xs;
    XInfo xi;
    xi.active = 1;
    xi.sw = -1;
    xi.xt = x;
    xi.jt = 63 - __clzll((long long)x);
    p1_unit<R, HI, false>(a.psi, xi, rho, a.ring + ((size_t)(t % 3) * a.X + xs) * xlen, sm, lane, pre);
  }
  wait_prior_grid();  // every CTA waits before it exits (transitive ordering of the chain)
}

// moment slots the stage kernels need: one per warp of a full-occupancy grid
size_t adj_stage_slots(const hm_ctx *c) { return (size_t)c->num_sms * 8 * ADJ_WARPS; }

template <int HI, int QA>
int launch_adj_stages(hm_ctx *c, const AdjStageArgs &a0, int *nwarps_out) {
  AdjStageArgs a = a0;
  const size_t smem = (size_t)ADJ_WARPS * 32 * R * sizeof(double2);
  HM_CUDA(c, cudaFuncSetAttribute(k_adjs_p1<HI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  HM_CUDA(c, cudaFuncSetAttribute(k_adjs_p2f<HI, QA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  HM_CUDA(c, cudaFuncSetAttribute(k_adjs_p1b<HI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0, occ_g = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_adjs_p2f<HI, QA>, ADJ_WARPS * 32, smem));
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_g, k_adjs_grad, GRAD_WARPS * 32, 0));
  occ = std::max(1, std::min(occ, 8));
  occ_g = std::max(1, occ_g);
  const int blocks = c->num_sms * occ, blocks_g = c->num_sms * occ_g;
  const int nw = blocks * ADJ_WARPS;
  HM_TRY(ensure_dev(c, (void **)&c->d_ctrl, &c->ctrl_cap, 4 * sizeof(unsigned)));
  HM_CUDA(c, cudaMemsetAsync(c->d_ctrl, 0, 4 * sizeof(unsigned), c->stream));
  a.stage = c->d_ctrl;
  const int nst = a.nbatch + 3;
  const int G = std::min(nst, 32);
  // stage s, kind k: one chained launch (the very first waits for everything before it)
  auto launch = [&](int s, int kind) {
    a.node = s;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(kind == 0 ? blocks_g : blocks);
    lc.blockDim = dim3((kind == 0 ? GRAD_WARPS : ADJ_WARPS) * 32);
    lc.dynamicSmemBytes = kind == 0 ? 0 : smem;
    lc.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = (s > 0 || kind > 0) ? 1 : 0;
    switch (kind) {
      case 0: return cudaLaunchKernelEx(&lc, k_adjs_grad, a);
      case 1: return cudaLaunchKernelEx(&lc, k_adjs_p1b<HI>, a);
      case 2: return cudaLaunchKernelEx(&lc, k_adjs_p2f<HI, QA>, a);
      default: return cudaLaunchKernelEx(&lc, k_adjs_p1<HI>, a);
    }
  };
  cudaError_t ce = cudaSuccess;
  if (nst <= G) {
    // a short sweep: direct launches cost less host time than capturing a graph
    for (int s = 0; s < nst && ce == cudaSuccess; ++s)
      for (int kind = 0; kind < 4 && ce == cudaSuccess; ++kind) ce = launch(s, kind);
    c->launches += 4 * nst;
    if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "adjoint launch failed: %s", cudaGetErrorString(ce));
    *nwarps_out = nw;
    return HM_OK;
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  HM_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  for (int s = 0; s < G && ce == cudaSuccess; ++s)
    for (int kind = 0; kind < 4 && ce == cudaSuccess; ++kind) ce = launch(s, kind);
  if (ce == cudaSuccess) {
    k_stage_advance<<<1, 1, 0, c->stream>>>(a.stage, (unsigned)G);
    ce = cudaGetLastError();
  }
  const cudaError_t ce_end = cudaStreamEndCapture(c->stream, &graph);
  if (ce == cudaSuccess) ce = ce_end;
  if (ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return set_err(c, HM_ERR_CUDA, "adjoint graph capture failed: %s", cudaGetErrorString(ce));
  }
  ce = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess)
    return set_err(c, HM_ERR_CUDA, "adjoint graph instantiation failed: %s", cudaGetErrorString(ce));
  for (int s = 0; s < nst && ce == cudaSuccess; s += G) {
    ce = cudaGraphLaunch(exec, c->stream);
    c->launches += 4 * G + 1;
  }
  cudaGraphExecDestroy(exec);
  if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "adjoint graph launch failed: %s", cudaGetErrorString(ce));
  *nwarps_out = nw;
  return HM_OK;
}

int run_adj_stages(hm_ctx *c, const double2 *psi, int n, int q, double2 *grad, double *mpart, int *nw) {
  const uint64_t len = 1ull << n, xlen = len / 2;
  AdjStageArgs a;
  memset(&a, 0, sizeof a);
  a.psi = psi;
  a.grad = grad;
  a.q = q;
  a.n = n;
  a.cq = 2.0 * q * pow(4.0, q);
  a.q4 = pow(4.0, q);
  a.x_begin = 1u << PB;
  // Batch size: from HM_PARAM_ADJ_BATCH, else measured on B200 (time of hm_sre_grad over
  // that of hm_sre, q = 2; the stages are fixed-cost, which favours large batches until
  // the ring + Gamma working set, 5 X 2^(n-1) complex, costs more than it saves):
  //   n = 14: X = 1024 2.80 (128 .. 512: 3.1)    n = 16: X = 512 2.53 (128: 2.96)
  //   n = 17: X = 512 2.80 (128: 3.06)           n = 18: X = 512 2.92 (128: 3.12)
  //   n = 19: X = 128 3.00 (32: 3.08)            n = 20: X = 64 2.90 (32: 2.95, 128: 3.13)
  //   n = 21: X = 8 3.90 (4: 4.49, 16: 4.17, 64: 5.64)
  // X <= 2^PB keeps every batch aligned inside one pairing-bit class (and divides the
  // 2^n - 2^PB X-strings); the working set stays within 8 GiB.
  uint64_t X = twopass_cfg().adj_x > 0 ? (uint64_t)twopass_cfg().adj_x
                                       : (n <= 15 ? 1024 : n <= 18 ? 512 : n == 19 ? 128 : n == 20 ? 64 : 8);
  if (X > (1u << PB)) X = 1u << PB;
  while (X > 1 && 5 * X * xlen * sizeof(double2) > ((uint64_t)8 << 30)) X >>= 1;
  if (X > len - a.x_begin) X = len - a.x_begin;
  a.X = (int)X;
  a.nbatch = (int)((len - a.x_begin) / X);
  // X-string groups per gradient row: enough units for about four per gradient warp, so
  // that the chain of dependent loads of one unit (X / ng X-strings) stays short at small
  // n; at most 8 groups (each adds one partial gradient to write and fold)
  const long long units = 2LL * GPARTS * (long long)(xlen >> PB);
  const long long target = 4LL * c->num_sms * GRAD_CTAS * GRAD_WARPS;
  int ng = 1;
  while (ng < 8 && (uint64_t)(2 * ng) * GX <= X && units * ng < target) ng *= 2;
  a.ng = ng;
  HM_TRY(ensure_dev(c, &c->d_aux, &c->aux_cap, (5 * X * xlen + (size_t)(ng - 1) * len) * sizeof(double2)));
  a.ring = (double2 *)c->d_aux;
  a.gam = a.ring + 3 * X * xlen;
  a.gpart = a.gam + 2 * X * xlen;
  if (ng > 1) HM_CUDA(c, cudaMemsetAsync(a.gpart, 0, (size_t)(ng - 1) * len * sizeof(double2), c->stream));
  a.mpart = mpart;  // zeroed by the caller, one slot per warp (adj_stage_slots)
  int r = HM_ERR_SIZE;
  switch (n - 1 - PB) {
#define HM_ADJS(HIv)                                                                     \
  case HIv:                                                                              \
    r = q == 2 ? launch_adj_stages<HIv, 2>(c, a, nw)                                     \
               : (q == 3 ? launch_adj_stages<HIv, 3>(c, a, nw) : launch_adj_stages<HIv, 0>(c, a, nw)); \
    break;
    HM_ADJS(1)
    HM_ADJS(2)
    HM_ADJS(3)
    HM_ADJS(4)
    HM_ADJS(5)
    HM_ADJS(6)
    HM_ADJS(7)
    HM_ADJS(8)
    HM_ADJS(9)
    HM_ADJS(10)
#undef HM_ADJS
    default:
      break;
  }
  if (r == HM_OK && ng > 1) {
    k_adj_fold_groups<<<c->num_sms * 4, 256, 0, c->stream>>>(grad, a.gpart, ng - 1, len);
    c->launches += 1;
    HM_CUDA(c, cudaGetLastError());
  }
  return r;
}

}  // namespace

int run_sre_grad(hm_ctx *c, const double2 *psi, int n, int q, double *m_out, double2 *grad_dev) {
  AdjArgs a;
  memset(&a, 0, sizeof a);
  a.psi = psi;
  a.n = n;
  a.q = q;
  a.cq_x = 2.0 * q * pow(4.0, q);
  a.cq_0 = 2.0 * q;
  const uint64_t len = 1ull << n;
  // chunk: G of at most 1 GiB.  Each chunk costs four launches; with small chunks (16
  // X-strings at n = 18 for 64 MiB) the launches were under-filled and dominated the time
  int chunk = (int)std::max<uint64_t>(1, ((uint64_t)1 << 30) / (len * sizeof(double2)));
  if ((uint64_t)chunk > len) chunk = (int)len;
  if (n >= 12 && chunk > (1 << PB)) chunk = 1 << PB;  // the chunked kernels only see x < 2^PB
  a.chunk = chunk;
  HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, (size_t)chunk * len * sizeof(double2) +
                                                       (n >= 12 ? (size_t)chunk * (len / 2) * sizeof(double2) : 0)));
  a.G = (double2 *)c->d_inter;
  a.ring = a.G + (size_t)chunk * len;
  a.grad = grad_dev;
  HM_CUDA(c, cudaMemsetAsync(grad_dev, 0, len * sizeof(double2), c->stream));
  const size_t smem = 4 * 32 * R * sizeof(double2);
  int blocks;
  if (n <= 11) {
    blocks = (chunk + 3) / 4;
  } else {
    a.U = 1 << (n - 11);
    blocks = (int)(((long long)chunk * a.U + 3) / 4);
    HM_TRY(ensure_dev(c, &c->d_aux2, &c->aux2_cap, 10 * len * sizeof(double2)));
    k_psi_swapped<double2><<<c->num_sms * 8, 256, 0, c->stream>>>(psi, (double2 *)c->d_aux2, n, 10);
    c->launches += 1;
    for (int j = 0; j < 10; ++j) a.psi_sw[j] = (const double2 *)c->d_aux2 + (size_t)j * len;
  }
  const int nw = blocks * 4;
  // moment partials: the chunked kernels' warps, then one slot per warp of the stage kernels
  const size_t nslots = (size_t)nw + (n >= 12 ? adj_stage_slots(c) : 0);
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap, nslots * sizeof(double) + 64));
  HM_CUDA(c, cudaMemsetAsync(c->d_partials, 0, nslots * sizeof(double), c->stream));
  a.mpart = c->d_partials;
  const unsigned accb = (unsigned)std::min<uint64_t>((len + 31) / 32, (uint64_t)c->num_sms * 8);
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  // n >= 12: the chunked kernels cover x < 2^PB (relabelled copies, x = 0); the stage
  // kernels the rest
  const uint64_t x_chunked = n >= 12 ? std::min<uint64_t>(len, 1u << PB) : len;
  for (uint64_t x0 = 0; x0 < x_chunked; x0 += chunk) {
    a.x0 = x0;
    a.nx = (int)std::min<uint64_t>(chunk, x_chunked - x0);
    if (n <= 11) {
#define HM_ADJF(NBv)                                                                                  \
  case NBv:                                                                                           \
    cudaFuncSetAttribute(k_adj_fused<NBv>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
    k_adj_fused<NBv><<<blocks, 128, smem, c->stream>>>(a);                                            \
    break;
      switch (n - 1) {
        HM_ADJF(0)
        HM_ADJF(1)
        HM_ADJF(2)
        HM_ADJF(3)
        HM_ADJF(4)
        HM_ADJF(5)
        HM_ADJF(6)
        HM_ADJF(7)
        HM_ADJF(8)
        HM_ADJF(9)
        HM_ADJF(10)
        default:
          break;
      }
#undef HM_ADJF
    } else {
#define HM_ADJP(HIv)                                                                              \
  case HIv:                                                                                       \
    cudaFuncSetAttribute(k_adj_p1<HIv>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    cudaFuncSetAttribute(k_adj_p2<HIv>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    cudaFuncSetAttribute(k_adj_p1b<HIv>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    k_adj_p1<HIv><<<blocks, 128, smem, c->stream>>>(a);                                           \
    k_adj_p2<HIv><<<blocks, 128, smem, c->stream>>>(a);                                           \
    k_adj_p1b<HIv><<<blocks, 128, smem, c->stream>>>(a);                                          \
    break;
      switch (n - 11) {
        HM_ADJP(1)
        HM_ADJP(2)
        HM_ADJP(3)
        HM_ADJP(4)
        HM_ADJP(5)
        HM_ADJP(6)
        HM_ADJP(7)
        HM_ADJP(8)
        HM_ADJP(9)
        HM_ADJP(10)
        default:
          break;
      }
#undef HM_ADJP
    }
    k_adj_acc<<<accb, 32 * ACC_SEGS, 0, c->stream>>>(a);
    c->launches += n <= 11 ? 2 : 4;
  }
  HM_CUDA(c, cudaGetLastError());
  if (n >= 12 && len > x_chunked) {
    int nw_st = 0;
    HM_TRY(run_adj_stages(c, psi, n, q, grad_dev, c->d_partials + nw, &nw_st));
  }
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, sizeof(double) * 16));
  k_adj_finish<<<1, 256, 0, c->stream>>>(grad_dev, len, a.mpart, (int)nslots, c->d_out);
  c->launches += 1;
  HM_TRY(ensure_host(c, (void **)&c->h_out, &c->h_out_cap, sizeof(double) * 24));
  HM_CUDA(c, cudaMemcpyAsync(c->h_out, c->d_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  *m_out = c->h_out[0];
  return HM_OK;
}

}  // namespace hm

extern "C" int hm_sre_grad(hm_ctx *c, const double *psi, int n, double q, double *out_sre, double *grad) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!psi || !out_sre || !grad) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  if (n < 1 || n > 21) return hm::set_err(c, HM_ERR_SIZE, "adjoint: n = %d outside [1, 21]", n);
  if (!(q == floor(q) && q >= 1.0 && q <= 8.0))
    return hm::set_err(c, HM_ERR_Q, "adjoint: q = %g must be an integer in [1, 8]", q);
  HM_CUDA(c, cudaSetDevice(c->device));
  c->launches = 0;
  const size_t len = (size_t)1 << n;
  HM_TRY(hm::ensure_dev(c, &c->d_psi, &c->psi_cap, 2 * len * sizeof(double2)));
  double2 *dpsi = (double2 *)c->d_psi, *dgrad = dpsi + len;
  HM_CUDA(c, cudaMemcpyAsync(dpsi, psi, len * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  double m = 0.0;
  HM_TRY(hm::run_sre_grad(c, dpsi, n, (int)q, &m, dgrad));
  HM_CUDA(c, cudaMemcpyAsync(grad, dgrad, len * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  *out_sre = -log2(m / (double)len);
  return HM_OK;
}
