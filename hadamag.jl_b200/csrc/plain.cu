// plain.cu -- the reference CUDA backend's launch structure, restated in CUDA C.
//
// This is the "plain GPU form" the fused kernels are measured against, and the path for
// n > 21.  It follows ext/HadaMAGCUDAExt.jl:1307-1410 (compute_chunk_sre_cuda_batched!
// and SRE): per batch of B = 128 X-strings the host walks the Gray code, uploads the
// masks, then launches
//   build            (ext/HadaMAGCUDAExt.jl:226-250)  g[i,b] = muladd(re_i, re_j+im_j, im_i*(im_j-re_j))
//   head             (46-97)   first min(10, n) stages of every 1024-element tile in smem
//   stage x (n-11)   (279-304) one radix-2 stage in global memory per launch
//   last + reduce    (484-674) last stage with per-thread Kahan sums, block tree, partials
//   (or reduce_cols  (401-482, 815-891) when the head already finished the transform)
// and folds the per-block partials into two scalars read back by the host every batch
// (1374-1375).  FP64 throughout.
#include <math.h>

#include <vector>

#include "hm_common.cuh"
#include "hm_ctx.h"

namespace hm {

constexpr int PLAIN_THREADS = 256;

static inline uint64_t gray_code_host(uint64_t k) { return k ^ (k >> 1); }

__global__ void k_plain_build(const double2 *__restrict__ psi, const uint64_t *__restrict__ masks,
                              double *__restrict__ X, uint64_t N) {
  const int b = blockIdx.y;
  const uint64_t mask = masks[b] & (N - 1);
  double *out = X + (size_t)b * N;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 zi = psi[i], zj = psi[i ^ mask];
    out[i] = fma(zi.x, zj.x + zj.y, zi.y * (zj.y - zj.x));
  }
}

__global__ void k_plain_head(double *__restrict__ X, uint64_t N, int tile, int fuse) {
  extern __shared__ double smh[];
  const int b = blockIdx.y;
  const uint64_t base = (uint64_t)blockIdx.x * tile;
  double *col = X + (size_t)b * N + base;
  for (int i = threadIdx.x; i < tile; i += blockDim.x) smh[i] = col[i];
  __syncthreads();
  for (int s = 0; s < fuse; ++s) {
    const int step = 1 << s;
    for (int k0 = threadIdx.x; k0 < (tile >> 1); k0 += blockDim.x) {
      const int group = k0 / step, offs = k0 % step;
      const int ai = group * (step << 1) + offs, bi = ai + step;
      const double a = smh[ai], c = smh[bi];
      smh[ai] = a + c;
      smh[bi] = a - c;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < tile; i += blockDim.x) col[i] = smh[i];
}

__global__ void k_plain_stage(double *__restrict__ X, uint64_t N, uint64_t s) {
  const int b = blockIdx.y;
  double *col = X + (size_t)b * N;
  const uint64_t half = N >> 1;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < half; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t group = k / s, offs = k % s;
    const uint64_t ai = group * (s << 1) + offs, bi = ai + s;
    const double a = col[ai], c = col[bi];
    col[ai] = a + c;
    col[bi] = a - c;
  }
}

__device__ __forceinline__ double plain_powq(double v2, double q, bool q2) { return q2 ? v2 * v2 : pow(v2, q); }

__device__ __forceinline__ void kahan(double &s, double &c, double v) {
  const double y = v - c;
  const double t = s + y;
  c = (t - s) - y;
  s = t;
}

// block tree of the four Kahan registers; out = s + c (as in the reference)
__device__ __forceinline__ void plain_block_reduce(double sp, double cp, double sm, double cm, double *out_p2,
                                                   double *out_mq) {
  extern __shared__ double smr[];
  const int nt = blockDim.x, t = threadIdx.x;
  smr[t] = sp;
  smr[t + nt] = cp;
  smr[t + 2 * nt] = sm;
  smr[t + 3 * nt] = cm;
  __syncthreads();
  for (int off = nt >> 1; off > 0; off >>= 1) {
    if (t < off) {
      smr[t] += smr[t + off];
      smr[t + nt] += smr[t + nt + off];
      smr[t + 2 * nt] += smr[t + 2 * nt + off];
      smr[t + 3 * nt] += smr[t + 3 * nt + off];
    }
    __syncthreads();
  }
  if (t == 0) {
    *out_p2 = smr[0] + smr[nt];
    *out_mq = smr[2 * nt] + smr[3 * nt];
  }
}

__global__ void k_plain_last_reduce(double *__restrict__ X, uint64_t N, uint64_t s, double *out_p2, double *out_mq,
                                    double q, int q2) {
  const int b = blockIdx.y;
  double *col = X + (size_t)b * N;
  const uint64_t half = N >> 1;
  double sp = 0, cp = 0, sm = 0, cm = 0;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < half; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t group = k / s, offs = k % s;
    const uint64_t ai = group * (s << 1) + offs, bi = ai + s;
    const double a = col[ai], c = col[bi];
    const double y = a + c, z = a - c;
    col[ai] = y;  // the reference writes the transformed values back
    col[bi] = z;
    const double y2 = y * y, z2 = z * z;
    kahan(sp, cp, y2);
    kahan(sp, cp, z2);
    kahan(sm, cm, plain_powq(y2, q, q2));
    kahan(sm, cm, plain_powq(z2, q, q2));
  }
  plain_block_reduce(sp, cp, sm, cm, out_p2 + (size_t)b * gridDim.x + blockIdx.x,
                     out_mq + (size_t)b * gridDim.x + blockIdx.x);
}

__global__ void k_plain_reduce_cols(const double *__restrict__ X, uint64_t N, double *out_p2, double *out_mq, double q,
                                    int q2) {
  const int b = blockIdx.y;
  const double *col = X + (size_t)b * N;
  const uint64_t nt = blockDim.x, g = nt * 2 * gridDim.x;
  double sp = 0, cp = 0, sm = 0, cm = 0;
  for (uint64_t i = blockIdx.x * (nt * 2) + threadIdx.x; i < N; i += g) {
    const double v1 = col[i], v1s = v1 * v1;
    kahan(sp, cp, v1s);
    kahan(sm, cm, plain_powq(v1s, q, q2));
    const uint64_t j = i + nt;
    if (j < N) {
      const double v2 = col[j], v2s = v2 * v2;
      kahan(sp, cp, v2s);
      kahan(sm, cm, plain_powq(v2s, q, q2));
    }
  }
  plain_block_reduce(sp, cp, sm, cm, out_p2 + (size_t)b * gridDim.x + blockIdx.x,
                     out_mq + (size_t)b * gridDim.x + blockIdx.x);
}

// device fold of one batch's partials (CUDA.sum in the reference)
__global__ void k_plain_batch_fold(const double *__restrict__ p2, const double *__restrict__ mq, int count,
                                   double *out) {
  __shared__ double a[256], bsh[256];
  double x = 0, y = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    x += p2[i];
    y += mq[i];
  }
  a[threadIdx.x] = x;
  bsh[threadIdx.x] = y;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      a[threadIdx.x] += a[threadIdx.x + o];
      bsh[threadIdx.x] += bsh[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = a[0];
    out[1] = bsh[0];
  }
}

static int plain_one_q(hm_ctx *c, const double2 *psi, int n, uint64_t kb, uint64_t ke, double q, double *p2_out,
                       double *m_out) {
  const uint64_t N = 1ull << n;
  const int L = n;
  int B = 128;
  while (B > 1 && (double)B * N * 8.0 > 16.0 * (1ull << 30)) B >>= 1;
  if ((uint64_t)B > ke - kb) B = (int)(ke - kb);
  if (B < 1) B = 1;
  const int threads = PLAIN_THREADS;
  const int blocks_x = (int)std::min<uint64_t>(1024, (N + threads * 2 - 1) / (threads * 2));
  HM_TRY(ensure_dev(c, &c->d_inter, &c->inter_cap, (size_t)B * N * sizeof(double)));
  const size_t part = (size_t)blocks_x * B;
  HM_TRY(ensure_dev(c, (void **)&c->d_partials, &c->partials_cap, sizeof(double) * 2 * part));
  HM_TRY(ensure_dev(c, &c->d_aux, &c->aux_cap, sizeof(uint64_t) * B));
  HM_TRY(ensure_dev(c, (void **)&c->d_out, &c->out_cap, sizeof(double) * 16));
  HM_TRY(ensure_host(c, &c->h_pin, &c->h_pin_cap, sizeof(uint64_t) * B));
  HM_TRY(ensure_host(c, (void **)&c->h_out, &c->h_out_cap, sizeof(double) * 16 + 64));
  double *X = (double *)c->d_inter;
  double *out_p2 = c->d_partials, *out_mq = c->d_partials + part;
  uint64_t *masks_h = (uint64_t *)c->h_pin, *masks_d = (uint64_t *)c->d_aux;
  const int tile_L = L < 10 ? L : 10;
  const int tile = 1 << tile_L, fuse = tile_L;
  const int q2 = (q == 2.0);
  double p2SAM = 0.0, mSAM = 0.0;
  uint64_t i = kb;
  while (i < ke) {
    int fill = 0;
    while (i < ke && fill < B) masks_h[fill++] = gray_code_host(i++);
    HM_CUDA(c, cudaMemcpyAsync(masks_d, masks_h, sizeof(uint64_t) * fill, cudaMemcpyHostToDevice, c->stream));
    dim3 gb((unsigned)std::min<uint64_t>((N + threads - 1) / threads, 65535), fill);
    k_plain_build<<<gb, threads, 0, c->stream>>>(psi, masks_d, X, N);
    dim3 gh((unsigned)(N / tile), fill);
    k_plain_head<<<gh, threads, tile * sizeof(double), c->stream>>>(X, N, tile, fuse);
    dim3 gr(blocks_x, fill);
    if (fuse == L) {
      k_plain_reduce_cols<<<gr, threads, 4 * threads * sizeof(double), c->stream>>>(X, N, out_p2, out_mq, q, q2);
    } else {
      for (int s = fuse; s <= L - 2; ++s) k_plain_stage<<<gr, threads, 0, c->stream>>>(X, N, 1ull << s);
      k_plain_last_reduce<<<gr, threads, 4 * threads * sizeof(double), c->stream>>>(X, N, 1ull << (L - 1), out_p2,
                                                                                    out_mq, q, q2);
    }
    c->launches += 3 + (fuse == L ? 0 : (L - 1 - fuse));
    HM_CUDA(c, cudaGetLastError());
    k_plain_batch_fold<<<1, 256, 0, c->stream>>>(out_p2, out_mq, blocks_x * fill, c->d_out);
    c->launches += 1;
    HM_CUDA(c, cudaMemcpyAsync(c->h_out, c->d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HM_CUDA(c, cudaStreamSynchronize(c->stream));  // per-batch host fold, as the reference
    p2SAM += c->h_out[0];
    mSAM += c->h_out[1];
  }
  *p2_out = p2SAM;
  *m_out = mSAM;
  return HM_OK;
}

int run_sre_plain(hm_ctx *c, const double2 *psi, int n, uint64_t kb, uint64_t ke, const QReq &q, double *out_dd) {
  if (n < 0 || n > 26) return set_err(c, HM_ERR_SIZE, "plain path: n = %d out of range [0, 26]", n);
  HM_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  for (int t = 0; t < q.nq; ++t) {
    double p2 = 0.0, m = 0.0;
    HM_TRY(plain_one_q(c, psi, n, kb, ke, q.q[t], &p2, &m));
    if (t == 0) {
      out_dd[0] = p2;
      out_dd[1] = 0.0;
    }
    out_dd[2 + 2 * t] = m;
    out_dd[3 + 2 * t] = 0.0;
  }
  HM_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HM_CUDA(c, cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  HM_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  return HM_OK;
}

}  // namespace hm
