// stateprep.cu -- state preparation on the device: two-site gates, brick-wall circuits of
// them, and reduced density matrices.  These produce the inputs of the SRE and Mana paths
// (rand_haar / apply_2gate! of src/State.jl:111-345, reduced_density_matrix of
// src/DensityMatrix.jl:94-123), which the reference runs as scalar host loops.
//
// Conventions (the reference's): sites are 1-based, site 1 the least significant digit
// of the linear index; a two-site gate is a q^2 x q^2 matrix in column-major order whose
// row / column index is o = o1 q + o2 / in = d1 q + d2, with d1 the digit of site s1.
#include <math.h>

#include <vector>

#include "hm_ctx.h"
#include "hm_common.cuh"

namespace hm {

namespace {

// gate in row-major order, g[o * q^2 + in]
struct Gate2 {
  double2 g[81];
};

// One thread per group of q^2 amplitudes that the gate mixes (the indices whose digits at
// sites s1, s2 run over all values): gather, multiply, scatter in place.  Every amplitude
// belongs to exactly one group, so the in-place update needs no second buffer.
template <int Q>
__global__ void k_apply_2gate(double2 *__restrict__ psi, uint64_t ngroups, uint64_t p1, uint64_t p2, uint64_t plo,
                              uint64_t pmid, const __grid_constant__ Gate2 G) {
  constexpr int Q2 = Q * Q;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ngroups;
       t += (uint64_t)gridDim.x * blockDim.x) {
    // base index: t with a zero digit inserted at the lower and at the higher site
    uint64_t base;
    if constexpr (Q == 2) {
      const uint64_t lo = t & (plo - 1), rest = t / plo;
      const uint64_t mid = rest & (pmid - 1), hi = rest / pmid;
      base = lo + plo * 2 * (mid + pmid * 2 * hi);
    } else {
      const uint64_t lo = t % plo, rest = t / plo;
      const uint64_t mid = rest % pmid, hi = rest / pmid;
      base = lo + plo * Q * (mid + pmid * Q * hi);
    }
    double2 a[Q2];
#pragma unroll
    for (int in = 0; in < Q2; ++in) a[in] = psi[base + (in / Q) * p1 + (in % Q) * p2];
#pragma unroll
    for (int o = 0; o < Q2; ++o) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int in = 0; in < Q2; ++in) {
        const double2 g = G.g[o * Q2 + in];
        re = fma(g.x, a[in].x, fma(-g.y, a[in].y, re));
        im = fma(g.x, a[in].y, fma(g.y, a[in].x, im));
      }
      psi[base + (o / Q) * p1 + (o % Q) * p2] = make_double2(re, im);
    }
  }
}

inline uint64_t upow(int q, int e) {
  uint64_t r = 1;
  for (int k = 0; k < e; ++k) r *= (uint64_t)q;
  return r;
}

int launch_2gate(hm_ctx *c, double2 *psi, int n, int q, const double *gate_colmajor, int s1, int s2) {
  Gate2 G;
  const int q2 = q * q;
  for (int o = 0; o < q2; ++o)
    for (int in = 0; in < q2; ++in)
      G.g[o * q2 + in] = make_double2(gate_colmajor[2 * (o + q2 * in)], gate_colmajor[2 * (o + q2 * in) + 1]);
  const int lo = (s1 < s2 ? s1 : s2) - 1, hi = (s1 < s2 ? s2 : s1) - 1;
  const uint64_t N = upow(q, n), ngroups = N / (uint64_t)q2;
  const uint64_t p1 = upow(q, s1 - 1), p2 = upow(q, s2 - 1), plo = upow(q, lo), pmid = upow(q, hi - lo - 1);
  const uint64_t want = (ngroups + 255) / 256;
  const unsigned blocks = (unsigned)std::min<uint64_t>(std::max<uint64_t>(want, 1), (uint64_t)c->num_sms * 16);
  if (q == 2)
    k_apply_2gate<2><<<blocks, 256, 0, c->stream>>>(psi, ngroups, p1, p2, plo, pmid, G);
  else
    k_apply_2gate<3><<<blocks, 256, 0, c->stream>>>(psi, ngroups, p1, p2, plo, pmid, G);
  c->launches += 1;
  HM_CUDA(c, cudaGetLastError());
  return HM_OK;
}

// ---------------------------------------------------------------------------------
// rho_A[i, j] = sum_k A(i, k) conj(A(j, k)),  A(i, k) = psi[i + dimA k] (left) or
// psi[i dimB + k] (right); column-major output.  64 x 64 output tiles, 256 threads with
// 4 x 4 outputs each (16 complex multiply-adds per 8 shared-memory loads), k in slices
// of 16 through shared memory.  blockIdx.z splits k into `nsplit` ranges whose partial
// tiles are summed afterwards in split order.
constexpr int RT = 64, RK = 16;

__global__ void __launch_bounds__(256, 2) k_rdm(const double2 *__restrict__ psi, uint64_t dimA, uint64_t dimB, int side,
                                             uint64_t k_per_split, double2 *__restrict__ out) {
  __shared__ double2 As[RT][RK + 1], Bs[RT][RK + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const uint64_t i0 = (uint64_t)blockIdx.x * RT, j0 = (uint64_t)blockIdx.y * RT;
  const uint64_t kb = (uint64_t)blockIdx.z * k_per_split;
  const uint64_t ke = kb + k_per_split < dimB ? kb + k_per_split : dimB;
  double2 acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int w = 0; w < 4; ++w) acc[u][w] = make_double2(0.0, 0.0);
  for (uint64_t k0 = kb; k0 < ke; k0 += RK) {
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int e = threadIdx.x + 256 * h;  // element of the 64 x 16 slice
      // fast index along consecutive addresses: rows on the left, k on the right
      const int r = side == 0 ? (e & 63) : (e >> 4), kk = side == 0 ? (e >> 6) : (e & 15);
      const uint64_t k = k0 + kk;
      const uint64_t ia = i0 + r, ja = j0 + r;
      double2 va = make_double2(0.0, 0.0), vb = make_double2(0.0, 0.0);
      if (k < ke) {
        if (ia < dimA) va = psi[side == 0 ? ia + dimA * k : ia * dimB + k];
        if (ja < dimA) vb = psi[side == 0 ? ja + dimA * k : ja * dimB + k];
      }
      As[r][kk] = va;
      Bs[r][kk] = vb;
    }
    __syncthreads();
#pragma unroll 2
    for (int kk = 0; kk < RK; ++kk) {
      double2 a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = As[tx + 16 * u][kk];
        b[u] = Bs[ty + 16 * u][kk];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w) {  // a conj(b)
          acc[u][w].x = fma(a[u].x, b[w].x, fma(a[u].y, b[w].y, acc[u][w].x));
          acc[u][w].y = fma(a[u].y, b[w].x, fma(-a[u].x, b[w].y, acc[u][w].y));
        }
    }
    __syncthreads();
  }
  double2 *o = out + (size_t)blockIdx.z * dimA * dimA;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const uint64_t i = i0 + tx + 16 * u, j = j0 + ty + 16 * w;
      if (i < dimA && j < dimA) o[i + dimA * j] = acc[u][w];
    }
}

__global__ void k_sum_splits(const double2 *__restrict__ part, uint64_t len, int nsplit, double2 *__restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    double2 s = part[i];
    for (int k = 1; k < nsplit; ++k) {
      const double2 p = part[(size_t)k * len + i];
      s.x += p.x;
      s.y += p.y;
    }
    out[i] = s;
  }
}

int check_state(hm_ctx *c, int n, int q) {
  if (q != 2 && q != 3) return set_err(c, HM_ERR_ARG, "only q = 2 and q = 3 are implemented (got q = %d)", q);
  const int nmax = q == 2 ? 30 : 19;
  if (n < 1 || n > nmax) return set_err(c, HM_ERR_SIZE, "n = %d outside [1, %d] for q = %d", n, nmax, q);
  return HM_OK;
}

}  // namespace

}  // namespace hm

extern "C" {

int hm_apply_2gate(hm_ctx *c, double *psi, int n, int q, const double *gate, int s1, int s2) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!psi || !gate) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  HM_TRY(hm::check_state(c, n, q));
  if (n < 2 || s1 < 1 || s2 < 1 || s1 > n || s2 > n || s1 == s2)
    return hm::set_err(c, HM_ERR_ARG, "sites (%d, %d) must be two different sites in [1, %d]", s1, s2, n);
  HM_CUDA(c, cudaSetDevice(c->device));
  c->launches = 0;
  const size_t bytes = hm::upow(q, n) * sizeof(double2);
  HM_TRY(hm::ensure_dev(c, &c->d_psi, &c->psi_cap, bytes));
  HM_CUDA(c, cudaMemcpyAsync(c->d_psi, psi, bytes, cudaMemcpyHostToDevice, c->stream));
  HM_TRY(hm::launch_2gate(c, (double2 *)c->d_psi, n, q, gate, s1, s2));
  HM_CUDA(c, cudaMemcpyAsync(psi, c->d_psi, bytes, cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  return HM_OK;
}

int hm_brick_wall(hm_ctx *c, double *psi, int n, int q, int depth, const double *gates, int ngates) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!psi || (ngates > 0 && !gates)) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  HM_TRY(hm::check_state(c, n, q));
  if (depth < 0) return hm::set_err(c, HM_ERR_ARG, "depth = %d < 0", depth);
  long long expect = 0;
  for (int layer = 1; layer <= depth; ++layer)
    for (int s = (layer & 1) ? 1 : 2; s <= n - 1; s += 2) ++expect;
  if (expect != ngates)
    return hm::set_err(c, HM_ERR_ARG, "depth %d on %d sites takes %lld gates, got %d", depth, n, expect, ngates);
  HM_CUDA(c, cudaSetDevice(c->device));
  c->launches = 0;
  const size_t bytes = hm::upow(q, n) * sizeof(double2);
  const int q4 = q * q * q * q;
  HM_TRY(hm::ensure_dev(c, &c->d_psi, &c->psi_cap, bytes));
  HM_CUDA(c, cudaMemcpyAsync(c->d_psi, psi, bytes, cudaMemcpyHostToDevice, c->stream));
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  int k = 0;
  for (int layer = 1; layer <= depth; ++layer)
    for (int s = (layer & 1) ? 1 : 2; s <= n - 1; s += 2, ++k)
      HM_TRY(hm::launch_2gate(c, (double2 *)c->d_psi, n, q, gates + (size_t)2 * q4 * k, s, s + 1));
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_CUDA(c, cudaMemcpyAsync(psi, c->d_psi, bytes, cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  return HM_OK;
}

int hm_reduced_density_matrix(hm_ctx *c, const double *psi, int n, int q, int NA, int side, double *rho) {
  if (!c) return HM_ERR_ARG;
  c->err.clear();
  if (!psi || !rho) return hm::set_err(c, HM_ERR_ARG, "null pointer");
  HM_TRY(hm::check_state(c, n, q));
  if (NA < 0 || NA > n) return hm::set_err(c, HM_ERR_ARG, "need 0 <= NA <= N (got NA = %d, N = %d)", NA, n);
  if (side != 0 && side != 1) return hm::set_err(c, HM_ERR_ARG, "side must be 0 (left) or 1 (right)");
  const uint64_t dimA = hm::upow(q, NA), dimB = hm::upow(q, n - NA);
  if (dimA > 16384) return hm::set_err(c, HM_ERR_SIZE, "dim A = %llu above 16384", (unsigned long long)dimA);
  HM_CUDA(c, cudaSetDevice(c->device));
  c->launches = 0;
  const size_t bytes = hm::upow(q, n) * sizeof(double2);
  // split k so that about two CTAs per SM run, each over at least 256 values of k
  const uint64_t tiles = ((dimA + hm::RT - 1) / hm::RT) * ((dimA + hm::RT - 1) / hm::RT);
  uint64_t nsplit = std::max<uint64_t>(1, (2 * (uint64_t)c->num_sms + tiles - 1) / tiles);
  nsplit = std::min<uint64_t>(nsplit, std::max<uint64_t>(1, dimB / 256));
  nsplit = std::min<uint64_t>(nsplit, 1024);
  const uint64_t kps = ((dimB + nsplit - 1) / nsplit + hm::RK - 1) / hm::RK * hm::RK;
  nsplit = (dimB + kps - 1) / kps;
  const size_t out_bytes = dimA * dimA * sizeof(double2);
  HM_TRY(hm::ensure_dev(c, &c->d_psi, &c->psi_cap, bytes));
  HM_TRY(hm::ensure_dev(c, &c->d_aux, &c->aux_cap, out_bytes * (nsplit + 1)));
  HM_CUDA(c, cudaMemcpyAsync(c->d_psi, psi, bytes, cudaMemcpyHostToDevice, c->stream));
  double2 *part = (double2 *)c->d_aux, *out = part + nsplit * dimA * dimA;
  const dim3 grid((unsigned)((dimA + hm::RT - 1) / hm::RT), (unsigned)((dimA + hm::RT - 1) / hm::RT),
                  (unsigned)nsplit);
  hm::k_rdm<<<grid, 256, 0, c->stream>>>((const double2 *)c->d_psi, dimA, dimB, side, kps, part);
  hm::k_sum_splits<<<c->num_sms * 4, 256, 0, c->stream>>>(part, dimA * dimA, (int)nsplit, out);
  c->launches += 2;
  HM_CUDA(c, cudaGetLastError());
  HM_CUDA(c, cudaMemcpyAsync(rho, out, out_bytes, cudaMemcpyDeviceToHost, c->stream));
  HM_CUDA(c, cudaStreamSynchronize(c->stream));
  return HM_OK;
}

}  // extern "C"
