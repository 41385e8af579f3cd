// mana.cu -- qutrit Mana kernels.
//
// Pure states (src/Mana.jl:19-92, src/Backends/Threads.jl:223-271).  For every ternary
// X-string x the reference forms
//     v(r) = conj psi(r (+) x) * (psi((-r) (+) x) / 3^L)        ((+): digitwise addition mod 3)
// applies the qutrit Hadamard H3^{(x)L} (src/Helpers.jl:249-292) and sums |W|; the Mana
// is log2(S) / log2(3).  The sum over x does not depend on the order in which the
// X-strings are visited, so x runs over 0 .. 3^L - 1 directly.
//
// The 3^L-point transform is split like the exact-SRE sweep: the low `lo` digits of r
// form a contiguous row (pass 1: gather + build + transform in shared memory), the high
// `hi` digits a strided column (pass 2: transform + sum |W|).  Batches of X-strings keep
// the intermediate resident in L2.  FP64 throughout.
//
// Mixed states (src/Mana.jl:123-314): w = M^{(x)N} vec9(rho) leg by leg, then
// log2(sum |w| / 3^N).
#include <math.h>

#include "hm_common.cuh"
#include "hm_ctx.h"

namespace hm {

namespace {

__host__ __device__ inline int ipow3(int e) {
  int r = 1;
  for (int i = 0; i < e; ++i) r *= 3;
  return r;
}

// digitwise (a (+) b) and ((-a) (+) b) for numbers of `nd` base-3 digits
__device__ inline int tadd(int a, int b, int nd) {
  int r = 0, p = 1;
  for (int i = 0; i < nd; ++i) {
    r += ((a % 3 + b % 3) % 3) * p;
    a /= 3;
    b /= 3;
    p *= 3;
  }
  return r;
}
__device__ inline int tnegadd(int a, int b, int nd) {
  int r = 0, p = 1;
  for (int i = 0; i < nd; ++i) {
    r += (((3 - a % 3) % 3 + b % 3) % 3) * p;
    a /= 3;
    b /= 3;
    p *= 3;
  }
  return r;
}

// the reference's 3-point DFT (a, b, c) -> (a+b+c, a+w b+w^2 c, a+w^2 b+w c), w = e^{2 pi i/3}
__device__ __forceinline__ void dft3(double2 &a, double2 &b, double2 &c) {
  const double wr = -0.5, wi = 0.86602540378443864676;  // cos, sin of 2 pi / 3
  const double r0 = a.x + b.x + c.x, i0 = a.y + b.y + c.y;
  const double r1 = a.x + wr * (b.x + c.x) - wi * (b.y - c.y);
  const double i1 = a.y + wr * (b.y + c.y) + wi * (b.x - c.x);
  const double r2 = a.x + wr * (b.x + c.x) + wi * (b.y - c.y);
  const double i2 = a.y + wr * (b.y + c.y) - wi * (b.x - c.x);
  a = make_double2(r0, i0);
  b = make_double2(r1, i1);
  c = make_double2(r2, i2);
}

// Consecutive Mana launches are chained by programmatic dependent launch: a grid lets the
// next one be scheduled from its start, and every thread of the next grid waits for this
// one to finish (and its memory to be visible) right before its first dependent access,
// and in any case before it exits, so that a grid's completion implies its predecessors'.
__device__ __forceinline__ void mana_allow_next() { asm volatile("griddepcontrol.launch_dependents;" :::); }
__device__ __forceinline__ void mana_wait_prior() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__host__ __device__ constexpr int ipow3c(int e) { return e <= 0 ? 1 : 3 * ipow3c(e - 1); }

// Register blocks of the qutrit transform H3^{(x)ND} of one vector of 3^ND elements
// (ND <= 6).  T = 3^ND / E threads hold E = min(27, 3^ND) elements each, in two phases
// separated by one shared-memory exchange:
//   phase A: digits 0 .. A-1 (A = min(3, ND)); thread t holds e = t E + k in register k;
//   phase B: digits A .. ND-1 (B = ND - A <= 3); thread t holds e = j + 27 m for the
//            GB = 27 / 3^B values j = t + T s (s < GB) and m < 3^B, in register s 3^B + m.
// Every element crosses shared memory once per pass (written after phase A, read for
// phase B); each thread runs its radix-27 / radix-3^B butterflies in registers.
template <int ND> struct QBlock {
  static constexpr int N = ipow3c(ND);
  static constexpr int E = N >= 27 ? 27 : N;
  static constexpr int T = N / E;
  static constexpr int A = ND < 3 ? ND : 3;
  static constexpr int B = ND - A;
  static constexpr int MB = ipow3c(B);
  static constexpr int GB = 27 / MB;
};

// H3 over one digit of the register index (stride ST = 3^d): register i pairs with
// i + ST and i + 2 ST when digit d of i is 0 (every index is a compile-time constant
// after unrolling, so the block stays in registers)
template <int NREG, int ST>
__device__ __forceinline__ void h3_digit(double2 (&v)[NREG]) {
#pragma unroll
  for (int i = 0; i < NREG; ++i)
    if ((i / ST) % 3 == 0 && i + 2 * ST < NREG) dft3(v[i], v[i + ST], v[i + 2 * ST]);
}
// H3 over digits 0 .. ND-1 (ND <= 3) of the register index
template <int NREG, int ND>
__device__ __forceinline__ void h3_regs(double2 (&v)[NREG]) {
  static_assert(ND <= 3, "a register block spans at most three digits");
  if constexpr (ND >= 1) h3_digit<NREG, 1>(v);
  if constexpr (ND >= 2) h3_digit<NREG, 3>(v);
  if constexpr (ND >= 3) h3_digit<NREG, 9>(v);
}

constexpr int MANA_MAX_THREADS = 256;

// shape of the two-pass split for L = LO + HI qutrits: pass 1 transforms rows of
// RL = 3^LO elements (ROWS rows per CTA), pass 2 columns of RH = 3^HI elements (COLS
// adjacent columns per CTA, so that a warp's loads cover consecutive columns)
template <int LO, int HI> struct ManaShape {
  using QR = QBlock<LO>;
  using QC = QBlock<HI>;
  static constexpr int RL = ipow3c(LO), RH = ipow3c(HI);
  static constexpr int ROWS = (MANA_MAX_THREADS / QR::T > RH) ? RH : MANA_MAX_THREADS / QR::T;
  static constexpr int COLS = (MANA_MAX_THREADS / QC::T > RL) ? RL : MANA_MAX_THREADS / QC::T;
  static constexpr int NT1 = (ROWS * QR::T + 31) / 32 * 32;
  static constexpr int NT2 = (COLS * QC::T + 31) / 32 * 32;
  // pass-1 row stride in shared memory: VS = 1 (mod 8) elements, so that the eight
  // 16-byte accesses of a quarter warp (consecutive threads T rr + t) fall on distinct
  // bank groups in both phases (T is odd, T^2 = 1 mod 8)
  static constexpr int VS = RL + ((1 - RL % 8) + 8) % 8;
  static constexpr size_t SM1 = QR::B > 0 ? (size_t)ROWS * VS * 16 : 0;
  static constexpr size_t SM2 = QC::B > 0 ? (size_t)RH * COLS * 16 : 0;
};

struct ManaArgs {
  const double2 *psi;
  double2 *inter;  // batch x RH x RL
  double *slots;   // per pass-2 CTA slot: dd (2 doubles)
  int x0, nx;      // X-strings of this batch: x0 .. x0 + nx - 1
  double invdim;
};

// pass 1: rows [blockIdx.x * ROWS, ...) of X-string x0 + blockIdx.y: gather + build
// v(r) = conj psi(r (+) x) psi((-r) (+) x) / 3^L, transform the row digits.  Pass 1 runs
// the block phases in the other order: phase A takes the HIGH three digits, thread t
// holding e = t + T k (so a warp's gathers for one k are adjacent elements), and phase B
// the low B digits in contiguous groups, thread t holding e = m + MB (t + T s).  The row
// is stored in the threads' order, position p = (s MB + m) T + t for register s MB + m:
// a fixed permutation of the positions, which pass 2 (columns) and the sum of |W| do not
// see, and which makes every store instruction of a warp contiguous.
template <int LO, int HI>
__global__ void __launch_bounds__(MANA_MAX_THREADS, 2) k_mana_p1(ManaArgs a) {
  using S = ManaShape<LO, HI>;
  using Q = typename S::QR;
  constexpr int RL = S::RL, RH = S::RH, ROWS = S::ROWS, E = Q::E, T = Q::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2 *sm = reinterpret_cast<double2 *>(smraw);  // ROWS x VS (phase-B exchange)
  constexpr int VS = S::VS;
  mana_allow_next();
  const int xi = blockIdx.y;
  if (xi >= a.nx) {  // uniform across the CTA
    mana_wait_prior();
    return;
  }
  const int x = a.x0 + xi;
  const int xL = x % RL, xH = x / RL;
  const int row0 = blockIdx.x * ROWS;
  const int nrows = min(ROWS, RH - row0);
  const int rr = threadIdx.x / T, t = threadIdx.x - rr * T;
  const bool act = rr < nrows;
  double2 v[E];
  if (act) {
    const int row = row0 + rr;
    const double2 *pa = a.psi + (size_t)tadd(row, xH, HI) * RL;
    const double2 *pb = a.psi + (size_t)tnegadd(row, xH, HI) * RL;
    // e = t + T k: the digit-wise e (+) xL and (-e) (+) xL split into the low B digits
    // (t, once per thread) and the A register digits of k, whose rotations by the digits
    // of xL are picked per register at compile time (no table, no shared-memory load)
    const int xlo = xL % T, xhi = xL / T;
    const int at = tadd(t, xlo, Q::B), nt = tnegadd(t, xlo, Q::B);
    int ra[3][3], rn[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int h = (xhi / ipow3c(i)) % 3;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ra[i][c] = ((h + c) % 3) * ipow3c(i) * T;
        rn[i][c] = ((h + 3 - c) % 3) * ipow3c(i) * T;
      }
    }
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const int k0 = k % 3, k1 = (k / 3) % 3, k2 = (k / 9) % 3;
      const int ia = at + ra[0][k0] + (Q::A > 1 ? ra[1][k1] : 0) + (Q::A > 2 ? ra[2][k2] : 0);
      const int in = nt + rn[0][k0] + (Q::A > 1 ? rn[1][k1] : 0) + (Q::A > 2 ? rn[2][k2] : 0);
      const double2 p = pa[ia];
      double2 q = pb[in];
      q.x *= a.invdim;
      q.y *= a.invdim;
      v[k] = make_double2(p.x * q.x + p.y * q.y, p.x * q.y - p.y * q.x);  // conj(p) * q
    }
    h3_regs<E, Q::A>(v);  // the register digits of k: element digits B .. LO-1
  }
  double2 *out = a.inter + ((size_t)xi * RH + row0 + rr) * RL;
  if constexpr (Q::B > 0) {
    if (act) {
#pragma unroll
      for (int k = 0; k < E; ++k) sm[rr * VS + t + T * k] = v[k];
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int s = 0; s < Q::GB; ++s)
#pragma unroll
        for (int m = 0; m < Q::MB; ++m) v[s * Q::MB + m] = sm[rr * VS + m + Q::MB * (t + T * s)];
      h3_regs<27, Q::B>(v);  // element digits 0 .. B-1
    }
    mana_wait_prior();  // the previous batch's pass 2 has read the intermediate
    if (act) {
#pragma unroll
      for (int r = 0; r < 27; ++r) out[r * T + t] = v[r];
    }
  } else {
    mana_wait_prior();
    if (act) {
#pragma unroll
      for (int k = 0; k < E; ++k) out[k] = v[k];
    }
  }
}

// pass 2: columns [blockIdx.x * COLS, ...) of X-string x0 + blockIdx.y: transform the
// column digits and add the CTA's sum |W| into its double-double slot
template <int LO, int HI>
__global__ void __launch_bounds__(MANA_MAX_THREADS, 2) k_mana_p2(ManaArgs a) {
  using S = ManaShape<LO, HI>;
  using Q = typename S::QC;
  constexpr int RL = S::RL, RH = S::RH, COLS = S::COLS, E = Q::E, T = Q::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2 *sm = reinterpret_cast<double2 *>(smraw);  // element e of column c at sm[e COLS + c]
  __shared__ double red[MANA_MAX_THREADS / 32];
  const int xi = blockIdx.y;
  const int c0 = blockIdx.x * COLS;
  const int ncols = min(COLS, RL - c0);
  const int t = threadIdx.x / COLS, c = threadIdx.x - t * COLS;
  const bool act = xi < a.nx && t < T && c < ncols;
  const double2 *in = a.inter + (size_t)xi * RH * RL + c0 + c;
  double2 v[E];
  mana_allow_next();
  mana_wait_prior();  // pass 1 of this batch has stored the intermediate
  if (act) {
#pragma unroll
    for (int k = 0; k < E; ++k) v[k] = in[(size_t)(t * E + k) * RL];
    h3_regs<E, Q::A>(v);
  }
  if constexpr (Q::B > 0) {
    if (act) {
#pragma unroll
      for (int k = 0; k < E; ++k) sm[(t * E + k) * COLS + c] = v[k];
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int s = 0; s < Q::GB; ++s)
#pragma unroll
        for (int m = 0; m < Q::MB; ++m) v[s * Q::MB + m] = sm[(t + T * s + 27 * m) * COLS + c];
      h3_regs<27, Q::B>(v);
    }
  }
  double sum = 0.0;
  if (act) {
#pragma unroll
    for (int k = 0; k < E; ++k) sum += sqrt(fma(v[k].x, v[k].x, v[k].y * v[k].y));
  }
  // warp sums, then the warps' sums in warp order
  sum = warp_sum(sum);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
    double *slot = a.slots + 2 * ((size_t)blockIdx.y * gridDim.x + blockIdx.x);
    dd acc{slot[0], slot[1]};
    dd_add(acc, tot);
    slot[0] = acc.hi;
    slot[1] = acc.lo;
  }
}

__global__ void k_fold_dd(const double *slots, int nslots, double *out) {
  __shared__ dd sh[256];
  dd acc{0.0, 0.0};
  for (int i = threadIdx.x; i < nslots; i += blockDim.x) dd_add_dd(acc, dd{slots[2 * i], slots[2 * i + 1]});
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) dd_add_dd(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sh[0].hi;
    out[1] = sh[0].lo;
  }
}

// ---------------------------------------------------------------------------------
// mixed states
struct M9 {
  double2 m[81];
};

// vec9 (src/Mana.jl:190-228): v[p] = rho[r0 + dim * c0], the base-9 digit of p for site k
// (site 1 most significant) being 3 i_k + j_k with i_k / j_k the k-th most significant
// ternary digits of r0 / c0
__global__ void k_vec_rho(const double2 *__restrict__ rho, double2 *__restrict__ v, int N, int dim, int op) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < op; p += gridDim.x * blockDim.x) {
    int t = p, r0 = 0, c0 = 0, w = 1;
    for (int k = 0; k < N; ++k) {  // least significant base-9 digit first = site N
      const int d9 = t % 9;
      t /= 9;
      r0 += (d9 / 3) * w;
      c0 += (d9 % 3) * w;
      w *= 3;
    }
    v[p] = rho[(size_t)r0 + (size_t)dim * c0];
  }
}

// one leg of M^{(x)N} (src/Mana.jl:236-281): y = M x on every fiber of stride 9^(N-leg)
__global__ void k_mana_leg(double2 *v, int op, int stride, M9 M) {
  const int nfib = op / 9;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nfib; f += gridDim.x * blockDim.x) {
    const int blk = f / stride, ofs = f % stride;
    const size_t base = (size_t)blk * stride * 9 + ofs;
    double2 x[9];
#pragma unroll
    for (int a = 0; a < 9; ++a) x[a] = v[base + (size_t)a * stride];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const double2 m = M.m[9 * r + c];
        sr += m.x * x[c].x - m.y * x[c].y;
        si += m.x * x[c].y + m.y * x[c].x;
      }
      v[base + (size_t)r * stride] = make_double2(sr, si);
    }
  }
}

__global__ void k_abs_sum_slots(const double2 *v, int len, double *slots) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) s += hypot(v[i].x, v[i].y);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    slots[2 * blockIdx.x] = red[0];
    slots[2 * blockIdx.x + 1] = 0.0;
  }
}

// host: the single-qutrit phase-point matrix of src/Mana.jl:123-182.  Row idx = 3a + a' is
// the column-major vec of A_u^T with A_u = T_u A0 T_u^dagger, T_{a,a'} = w^{(-2 a a') mod 3}
// Z^a X^{a'}, A0 = (1/3) sum_u T_u, X|k> = |k+1>, Z = diag(w^k).
struct C {
  double r, i;
};
static C cm(C a, C b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
static C ca(C a, C b) { return {a.r + b.r, a.i + b.i}; }
static void m3(const C *A, const C *B, C *out) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      C s{0, 0};
      for (int k = 0; k < 3; ++k) s = ca(s, cm(A[3 * i + k], B[3 * k + j]));
      out[3 * i + j] = s;
    }
}
static M9 phase_point_matrix() {
  const double PI = 3.14159265358979323846;
  const C w{cos(2 * PI / 3), sin(2 * PI / 3)};
  C X[9] = {}, Z[9] = {}, I[9] = {};
  const C wk[3] = {{1, 0}, w, cm(w, w)};
  for (int k = 0; k < 3; ++k) {
    X[3 * ((k + 1) % 3) + k] = {1, 0};
    Z[3 * k + k] = wk[k];
    I[3 * k + k] = {1, 0};
  }
  C Zp[3][9], Xp[3][9];
  for (int i = 0; i < 9; ++i) {
    Zp[0][i] = I[i];
    Zp[1][i] = Z[i];
    Xp[0][i] = I[i];
    Xp[1][i] = X[i];
  }
  m3(Z, Z, Zp[2]);
  m3(X, X, Xp[2]);
  C T[9][9];
  for (int a = 0; a < 3; ++a)
    for (int ap = 0; ap < 3; ++ap) {
      const int e = ((-2 * a * ap) % 3 + 3) % 3;
      C ph{1, 0};
      for (int t = 0; t < e; ++t) ph = cm(ph, w);
      C zx[9];
      m3(Zp[a], Xp[ap], zx);
      for (int i = 0; i < 9; ++i) T[3 * a + ap][i] = cm(ph, zx[i]);
    }
  C A0[9] = {};
  for (int u = 0; u < 9; ++u)
    for (int i = 0; i < 9; ++i) A0[i] = ca(A0[i], T[u][i]);
  for (int i = 0; i < 9; ++i) A0[i] = {A0[i].r / 3.0, A0[i].i / 3.0};
  M9 M;
  for (int u = 0; u < 9; ++u) {
    C Td[9], tmp[9], Au[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Td[3 * i + j] = {T[u][3 * j + i].r, -T[u][3 * j + i].i};
    m3(T[u], A0, tmp);
    m3(tmp, Td, Au);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M.m[9 * u + (i + 3 * j)] = make_double2(Au[3 * j + i].r, Au[3 * j + i].i);
  }
  return M;
}

}  // namespace

// one launch of a Mana pass, chained to the previous launch (chained = false for the
// first launch of a call, which waits for everything before it)
template <typename Kern>
static int mana_launch(hm_ctx *c, Kern kern, dim3 grid, int threads, size_t smem, const ManaArgs &a, bool chained) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = grid;
  lc.blockDim = dim3(threads);
  lc.dynamicSmemBytes = smem;
  lc.stream = c->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = chained ? 1 : 0;
  HM_CUDA(c, cudaLaunchKernelEx(&lc, kern, a));
  return HM_OK;
}

template <int LO, int HI>
static int run_mana_pure_t(hm_ctx *c, const double2 *psi, int xb, int xe, double *sum_dd) {
  using S = ManaShape<LO, HI>;
  constexpr int D = ipow3c(LO + HI);
  ManaArgs a;
  a.psi = psi;
  a.invdim = 1.0 / (double)D;
  const int g1 = (S::RH + S::ROWS - 1) / S::ROWS;
  const int g2 = (S::RL + S::COLS - 1) / S::COLS;
  auto k1 = k_mana_p1<LO, HI>;
  auto k2 = k_mana_p2<LO, HI>;
  HM_CUDA(c, cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SM1));
  HM_CUDA(c, cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SM2));
  int occ1 = 0, occ2 = 0;
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, k1, S::NT1, S::SM1));
  HM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k2, S::NT2, S::SM2));
  // X-strings per batch: whole waves of pass-1 CTAs (the last wave of a launch would
  // otherwise run partly empty), with the intermediate within 64 MiB (L2 resident)
  const int wave = c->num_sms * std::max(1, std::min(occ1, occ2));
  const size_t per_x = (size_t)D * sizeof(double2);
  const int bmax = (int)std::max<size_t>(1, ((size_t)64 << 20) / per_x);
  int B = std::min(bmax, std::max(1, wave / g1));
  for (int w = 2; (long long)w * wave / g1 <= bmax; ++w) B = (int)((long long)w * wave / g1);
  if (B > xe - xb) B = xe - xb;
  if (B > D) B = D;
  HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, (size_t)B * per_x));
  a.inter = (double2 *)c->d_inter;
  const size_t nslots = (size_t)g2 * B;
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap, nslots * 2 * sizeof(double)));
  HM_CUDA(c, cudaMemsetAsync(c->d_partials, 0, nslots * 2 * sizeof(double), c->stream));
  a.slots = c->d_partials;
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  for (int x0 = xb; x0 < xe; x0 += B) {
    a.x0 = x0;
    a.nx = std::min(B, xe - x0);
    HM_TRY(mana_launch(c, k1, dim3(g1, a.nx), S::NT1, S::SM1, a, x0 > xb));
    HM_TRY(mana_launch(c, k2, dim3(g2, B), S::NT2, S::SM2, a, true));
    c->launches += 2;
  }
  HM_CUDA(c, cudaGetLastError());
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, sizeof(double) * 16));
  k_fold_dd<<<1, 256, 0, c->stream>>>(c->d_partials, (int)nslots, c->d_out);
  c->launches += 1;
  HM_TRY(ensure_host(c, (void **)&c->h_out, &c->h_out_cap, sizeof(double) * 24));
  HM_CUDA(c, cudaMemcpyAsync(c->h_out, c->d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  sum_dd[0] = c->h_out[0];
  sum_dd[1] = c->h_out[1];
  return HM_OK;
}

// sum |W| over the X-strings [xb, xe) (natural order) as a double-double
int run_mana_pure(hm_ctx *c, const double2 *psi, int L, int xb, int xe, double *sum_dd) {
  // rows take the upper half of the digits: lo = ceil(L / 2), hi = L - lo
  switch (L) {
    case 1: return run_mana_pure_t<1, 0>(c, psi, xb, xe, sum_dd);
    case 2: return run_mana_pure_t<1, 1>(c, psi, xb, xe, sum_dd);
    case 3: return run_mana_pure_t<2, 1>(c, psi, xb, xe, sum_dd);
    case 4: return run_mana_pure_t<2, 2>(c, psi, xb, xe, sum_dd);
    case 5: return run_mana_pure_t<3, 2>(c, psi, xb, xe, sum_dd);
    case 6: return run_mana_pure_t<3, 3>(c, psi, xb, xe, sum_dd);
    case 7: return run_mana_pure_t<4, 3>(c, psi, xb, xe, sum_dd);
    case 8: return run_mana_pure_t<4, 4>(c, psi, xb, xe, sum_dd);
    case 9: return run_mana_pure_t<5, 4>(c, psi, xb, xe, sum_dd);
    case 10: return run_mana_pure_t<5, 5>(c, psi, xb, xe, sum_dd);
    case 11: return run_mana_pure_t<6, 5>(c, psi, xb, xe, sum_dd);
    case 12: return run_mana_pure_t<6, 6>(c, psi, xb, xe, sum_dd);
    default: return set_err(c, HM_ERR_SIZE, "L = %d qutrits outside [1, 12]", L);
  }
}

int run_mana_mixed(hm_ctx *c, const double2 *rho, int N, double *sum_dd) {
  const int dim = ipow3(N);
  int op = 1;
  for (int i = 0; i < N; ++i) op *= 9;
  HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, (size_t)op * sizeof(double2)));
  double2 *v = (double2 *)c->d_inter;
  const M9 M = phase_point_matrix();
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  const int blocks = std::max(1, std::min((op + 255) / 256, c->num_sms * 8));
  k_vec_rho<<<blocks, 256, 0, c->stream>>>(rho, v, N, dim, op);
  for (int leg = 1; leg <= N; ++leg) {
    int stride = 1;
    for (int i = 0; i < N - leg; ++i) stride *= 9;
    k_mana_leg<<<std::max(1, std::min((op / 9 + 127) / 128, c->num_sms * 8)), 128, 0, c->stream>>>(v, op, stride, M);
  }
  const int nb = std::max(1, std::min((op + 255) / 256, c->num_sms * 2));
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap, (size_t)nb * 2 * sizeof(double)));
  k_abs_sum_slots<<<nb, 256, 0, c->stream>>>(v, op, c->d_partials);
  HM_CUDA(c, cudaGetLastError());
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, sizeof(double) * 16));
  k_fold_dd<<<1, 256, 0, c->stream>>>(c->d_partials, nb, c->d_out);
  c->launches += 3 + N;  // vec9(rho), one per leg, the |w| sums, the fold
  HM_TRY(ensure_host(c, (void **)&c->h_out, &c->h_out_cap, sizeof(double) * 24));
  HM_CUDA(c, cudaMemcpyAsync(c->h_out, c->d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  sum_dd[0] = c->h_out[0];
  sum_dd[1] = c->h_out[1];
  return HM_OK;
}

}  // namespace hm

extern "C" {

int hm_mana_pure(hm_ctx *c, const double *psi, int L, double *out) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!psi || !out) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  if (L < 1 || L > 12) return hm::set_err(c, HM_ERR_SIZE, "L = %d qutrits outside [1, 12]", L);
  HM_CUDA(c, cudaSetDevice(c->device));
  c->launches = 0;
  const size_t D = (size_t)hm::ipow3(L);
  HM_TRY(hm::ensure_dev(c, &c->d_psi, &c->psi_cap, D * sizeof(double2)));
  HM_CUDA(c, cudaMemcpyAsync(c->d_psi, psi, D * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  double s[2];
  HM_TRY(hm::run_mana_pure(c, (const double2 *)c->d_psi, L, 0, (int)D, s));
  *out = log2(s[0] + s[1]) / log2(3.0);
  return HM_OK;
}

int hm_mana_pure_range(hm_ctx *c, const double *psi, int L, int64_t x_begin, int64_t x_end, double *sum_dd) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!psi || !sum_dd) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  if (L < 1 || L > 12) return hm::set_err(c, HM_ERR_SIZE, "L = %d qutrits outside [1, 12]", L);
  const int64_t D = hm::ipow3(L);
  if (x_begin < 0 || x_end > D || x_begin >= x_end)
    return hm::set_err(c, HM_ERR_ARG, "X-string range [%lld, %lld) outside [0, %lld)", (long long)x_begin,
                       (long long)x_end, (long long)D);
  HM_CUDA(c, cudaSetDevice(c->device));
  c->launches = 0;
  HM_TRY(hm::ensure_dev(c, &c->d_psi, &c->psi_cap, (size_t)D * sizeof(double2)));
  HM_CUDA(c, cudaMemcpyAsync(c->d_psi, psi, (size_t)D * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  return hm::run_mana_pure(c, (const double2 *)c->d_psi, L, (int)x_begin, (int)x_end, sum_dd);
}

int hm_mana_mixed(hm_ctx *c, const double *rho, int N, double *out) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!rho || !out) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  if (N < 1 || N > 8) return hm::set_err(c, HM_ERR_SIZE, "N = %d qutrits outside [1, 8]", N);
  HM_CUDA(c, cudaSetDevice(c->device));
  c->launches = 0;
  const size_t dim = (size_t)hm::ipow3(N);
  HM_TRY(hm::ensure_dev(c, &c->d_psi, &c->psi_cap, dim * dim * sizeof(double2)));
  HM_CUDA(c, cudaMemcpyAsync(c->d_psi, rho, dim * dim * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  double s[2];
  HM_TRY(hm::run_mana_mixed(c, (const double2 *)c->d_psi, N, s));
  *out = log2((s[0] + s[1]) / (double)dim);
  return HM_OK;
}

}  // extern "C"
