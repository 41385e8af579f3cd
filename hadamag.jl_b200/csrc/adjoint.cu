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
#include "sre_kernels.cuh"

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

__device__ __forceinline__ double powi(double y, int e) {
  double r = 1.0;
  for (int i = 0; i < e; ++i) r *= y;
  return r;
}

// pointwise map on every register: accumulate sum (W^2)^q, replace W by c W^{2q-1}
__device__ __forceinline__ double adj_pointwise(double2 (&v)[R], int q, double cq) {
  double m = 0.0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const double a = v[i].x, b = v[i].y;
    const double a2 = a * a, b2 = b * b;
    m += powi(a2, q) + powi(b2, q);
    v[i].x = cq * a * powi(a2, q - 1);
    v[i].y = cq * b * powi(b2, q - 1);
  }
  return m;
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
    mloc = adj_pointwise(v, qi, xz ? a.cq_0 : a.cq_x) * (xz ? 1.0 : pow_q_dev(4.0, a.q));
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
    mloc = adj_pointwise(v, (int)a.q, xz ? a.cq_0 : a.cq_x) * (xz ? 1.0 : pow_q_dev(4.0, a.q));
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

// grad(u) += sum over the chunk's X-strings of G_x(u) psi(u ^ x)
__global__ void k_adj_acc(AdjArgs a) {
  const uint64_t len = 1ull << a.n;
  for (uint64_t uu = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; uu < len; uu += (uint64_t)gridDim.x * blockDim.x) {
    double gr = 0.0, gi = 0.0;
    for (int xi = 0; xi < a.nx; ++xi) {
      const double2 g = a.G[(size_t)xi * len + uu];
      const double2 p = __ldg(a.psi + (uu ^ (a.x0 + xi)));
      gr += g.x * p.x - g.y * p.y;
      gi += g.x * p.y + g.y * p.x;
    }
    double2 o = a.grad[uu];
    o.x += gr;
    o.y += gi;
    a.grad[uu] = o;
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
// rH, sH of every rho; only the low bits xs of x differ).  Stage t runs
//   gradient units of batch t-3 (row rho, kind A/B, quarter of the row),
//   forward high + pointwise + backward high of batch t-1 (in place in the ring),
//   backward low of batch t-2 (Gamma rows, natural element order, into `gam`),
//   pass 1 of batch t,
// with the ring in 3 slots and `gam` in 2.  A gradient unit owns its rows and quarter
// for the whole batch: kind A adds sum_xs conj(Gamma_xs(e)) psi_sH(e ^ xL) to row rH,
// kind B adds sum_xs Gamma_xs(e) psi_rH(e) to row sH at e ^ xL (gathered at the permuted
// source positions).  No two units of a stage touch the same gradient entry and each
// entry's sum runs in a fixed order.
constexpr int ADJ_WARPS = 4;

struct AdjStageArgs {
  const double2 *psi;
  double2 *ring;    // 3 slots x X x 2^(n-1), tile-major (pass-1 layout)
  double2 *gam;     // 2 slots x X x 2^(n-1), Gamma rows in natural element order
  double2 *grad;    // 2^n, unscaled dm/dpsi
  double *mpart;    // per warp: sum of its pointwise-unit moments, over all stages
  unsigned *stage;  // [0] stage index, [1] CTAs finished in the current stage
  uint64_t x_begin;
  double cq, q4;    // c_q and 4^q for x != 0
  int q, n, X, nbatch;
};

// Gradient unit: destination elements p = 32 i + lane, i in [part * GU_REGS, +GU_REGS),
// of row rH (kind 0) or row sH (kind 1) of batch b.  Every X-string of the batch adds
//   kind 0:  conj(Gamma_x(p)) psi(sH, p ^ xL)       (grad at u1 = rH p)
//   kind 1:  Gamma_x(p ^ xL)  psi(rH, p ^ xL)       (grad at u2 = sH p)
// gathered at permuted addresses (no shuffles), four X-strings' loads in flight at once,
// summed in the order of xs.
constexpr int GU_REGS = 4;
constexpr int GU_PARTS = R / GU_REGS;  // units per row and kind

__device__ __forceinline__ void adj_grad_unit(const AdjStageArgs &a, long long b, uint64_t rho, int kind, int part,
                                              int lane) {
  const uint64_t xlen = 1ull << (a.n - 1);
  const uint64_t xb = a.x_begin + (uint64_t)b * a.X;  // aligned to X: xs occupies the low bits
  const int jt = 63 - __clzll((long long)xb);
  const uint64_t rH = insert0(rho, jt - PB), sH = rH ^ (xb >> PB);
  const uint32_t xLb = (uint32_t)(xb & ((1u << PB) - 1u));
  const double2 *gam_b = a.gam + (size_t)(b & 1) * a.X * xlen + (rho << PB);
  const double2 *rowA = a.psi + (rH << PB), *rowB = a.psi + (sH << PB);
  double2 acc[GU_REGS];
#pragma unroll
  for (int j = 0; j < GU_REGS; ++j) acc[j] = make_double2(0.0, 0.0);
#pragma unroll 1
  for (int xs0 = 0; xs0 < a.X; xs0 += 4) {
    double2 g[4][GU_REGS], w[4][GU_REGS];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int xs = xs0 + u < a.X ? xs0 + u : xs0;  // X < 4: repeat a valid one, masked below
      const double2 *g_row = gam_b + (size_t)xs * xlen;
      const uint32_t xL = xLb | (uint32_t)xs;
#pragma unroll
      for (int j = 0; j < GU_REGS; ++j) {
        const uint32_t p = (uint32_t)((part * GU_REGS + j) * 32 + lane);
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
    for (int u = 0; u < 4; ++u) {
      if (xs0 + u >= a.X) break;
#pragma unroll
      for (int j = 0; j < GU_REGS; ++j) {
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
  double2 *row = a.grad + ((kind == 0 ? rH : sH) << PB);
#pragma unroll
  for (int j = 0; j < GU_REGS; ++j) {
    const uint32_t p = (uint32_t)((part * GU_REGS + j) * 32 + lane);
    double2 o = row[p];
    o.x += acc[j].x;
    o.y += acc[j].y;
    row[p] = o;
  }
}

template <int HI>
__global__ void __launch_bounds__(ADJ_WARPS * 32, 2) k_adj_stage(AdjStageArgs a) {
  constexpr int LOGC = PB - HI;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *sm = reinterpret_cast<double2 *>(smraw) + warp * 32 * R;
  const long long t = (long long)*(volatile unsigned *)a.stage;
  if (t > (long long)a.nbatch + 2) return;  // padding stages of the last graph replay
  const int gwarp = blockIdx.x * ADJ_WARPS + warp, nwarps = gridDim.x * ADJ_WARPS;
  const uint64_t U = 1ull << HI, xlen = 1ull << (a.n - 1);
  const long long per = (long long)a.X * (long long)U;
  const long long ng = (t >= 3 && t - 3 < a.nbatch) ? 2 * GU_PARTS * (long long)U : 0;
  const long long n2 = (t >= 1 && t - 1 < a.nbatch) ? per : 0;
  const long long nb = (t >= 2 && t - 2 < a.nbatch) ? per : 0;
  const long long n1 = (t < a.nbatch) ? per : 0;
  double mloc = 0.0;
  for (long long u = gwarp; u < ng + n2 + nb + n1; u += nwarps) {
    if (u < ng) {
      adj_grad_unit(a, t - 3, (uint64_t)(u / (2 * GU_PARTS)), (int)((u / GU_PARTS) & 1), (int)(u % GU_PARTS), lane);
      continue;
    }
    long long r = u - ng;
    if (r < n2) {
      // forward over the row bits, pointwise map, backward over the row bits
      const long long b = t - 1;
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
      mloc += adj_pointwise(v, a.q, a.cq) * a.q4;
      if constexpr (LOGC >= 5) {
        reg_wht<R, LOGC - 5, 5>(v);
      } else {
        reg_wht<R, LOGC, 5>(v);
        transpose_ba(v, sm, lane);
        reg_wht<R, 0, 5>(v);
      }
#pragma unroll
      for (int i = 0; i < R; ++i) __stcg(tp + i * 32 + lane, v[i]);
      continue;
    }
    r -= n2;
    if (r < nb) {
      // backward over the low bits of one row; Gamma in natural element order to `gam`
      const long long b = t - 2;
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
      continue;
    }
    r -= nb;
    {
      // pass 1 (forward over the low bits) of batch t
      const int xs = (int)(r % a.X);
      const uint64_t rho = (uint64_t)(r / a.X);
      const uint64_t x = a.x_begin + (uint64_t)t * a.X + xs;
      XInfo xi;
      xi.active = 1;
      xi.sw = -1;
      xi.xt = x;
      xi.jt = 63 - __clzll((long long)x);
      p1_unit<R, HI, false>(a.psi, xi, rho, a.ring + ((size_t)(t % 3) * a.X + xs) * xlen, sm, lane);
    }
  }
  mloc = warp_sum(mloc);
  if (lane == 0) a.mpart[gwarp] += mloc;
  // the last CTA of the stage advances the stage index for the next launch
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(a.stage + 1, 1u);
    if (done == gridDim.x - 1) {
      a.stage[1] = 0;
      a.stage[0] = (unsigned)(t + 1);
      __threadfence();
    }
  }
}

// moment slots the stage kernels need: one per warp of a full-occupancy grid
size_t adj_stage_slots(const hm_ctx *c) { return (size_t)c->num_sms * 8 * ADJ_WARPS; }

template <int HI>
int launch_adj_stages(hm_ctx *c, const AdjStageArgs &a0, int *nwarps_out) {
  AdjStageArgs a = a0;
  const size_t smem = (size_t)ADJ_WARPS * 32 * R * sizeof(double2);
  auto kern = k_adj_stage<HI>;
  HM_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, ADJ_WARPS * 32, smem));
  if (occ < 1) occ = 1;
  const int blocks = c->num_sms * occ;
  const int nw = blocks * ADJ_WARPS;
  HM_TRY(ensure_dev(c, (void **)&c->d_ctrl, &c->ctrl_cap, 4 * sizeof(unsigned)));
  HM_CUDA(c, cudaMemsetAsync(c->d_ctrl, 0, 4 * sizeof(unsigned), c->stream));
  a.stage = c->d_ctrl;
  const int nst = a.nbatch + 3;
  const int G = std::min(nst, 32);
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  HM_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  for (int s = 0; s < G; ++s) kern<<<blocks, ADJ_WARPS * 32, smem, c->stream>>>(a);
  cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
  if (ce != cudaSuccess) return set_err(c, HM_ERR_CUDA, "adjoint graph capture failed: %s", cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess)
    return set_err(c, HM_ERR_CUDA, "adjoint graph instantiation failed: %s", cudaGetErrorString(ce));
  for (int s = 0; s < nst && ce == cudaSuccess; s += G) ce = cudaGraphLaunch(exec, c->stream);
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
  // Every stage costs a fixed few microseconds, so the batch is large: X <= 128 (a
  // gradient unit walks the batch's X-strings in sequence) with ring + Gamma rows within
  // 2 GiB.  Measured on B200: n = 14 X = 32 -> 128 cut the time 2.4x, n = 18 X = 16 ->
  // 128 by 18 %, although the larger working set leaves L2.
  uint64_t X = 128;
  while (X > 1 && 5 * X * xlen * sizeof(double2) > ((uint64_t)2 << 30)) X >>= 1;
  if (X > len - a.x_begin) X = len - a.x_begin;
  a.X = (int)X;
  a.nbatch = (int)((len - a.x_begin) / X);
  HM_TRY(ensure_dev(c, &c->d_aux, &c->aux_cap, 5 * X * xlen * sizeof(double2)));
  a.ring = (double2 *)c->d_aux;
  a.gam = a.ring + 3 * X * xlen;
  a.mpart = mpart;  // zeroed by the caller, one slot per warp (adj_stage_slots)
  int r = HM_ERR_SIZE;
  switch (n - 1 - PB) {
#define HM_ADJS(HIv) \
  case HIv:          \
    r = launch_adj_stages<HIv>(c, a, nw); \
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
    for (int j = 0; j < 10; ++j) a.psi_sw[j] = (const double2 *)c->d_aux2 + (size_t)j * len;
  }
  const int nw = blocks * 4;
  // moment partials: the chunked kernels' warps, then one slot per warp of the stage kernels
  const size_t nslots = (size_t)nw + (n >= 12 ? adj_stage_slots(c) : 0);
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap, nslots * sizeof(double) + 64));
  HM_CUDA(c, cudaMemsetAsync(c->d_partials, 0, nslots * sizeof(double), c->stream));
  a.mpart = c->d_partials;
  const unsigned accb = (unsigned)std::min<uint64_t>((len + 255) / 256, (uint64_t)c->num_sms * 8);
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
    k_adj_acc<<<accb, 256, 0, c->stream>>>(a);
  }
  HM_CUDA(c, cudaGetLastError());
  if (n >= 12 && len > x_chunked) {
    int nw_st = 0;
    HM_TRY(run_adj_stages(c, psi, n, q, grad_dev, c->d_partials + nw, &nw_st));
  }
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, sizeof(double) * 16));
  k_adj_finish<<<1, 256, 0, c->stream>>>(grad_dev, len, a.mpart, (int)nslots, c->d_out);
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
