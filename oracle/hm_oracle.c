/*
 * hm_oracle.c -- CPU restatement of HadaMAG.jl's exact-SRE / MC_SRE / Mana hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
 * reference arm may load it.  The product (libhadamag_b200.so) never links it.
 *
 * Parity status: the Gray-code tables are pinned bit-exactly to the properties the
 * reference's own tests assert (test/Basis_test.jl:3-25, 70-88).  The reference holds
 * no golden SRE / Mana values (its tests are backend cross-checks on unseeded states,
 * test/SRE_test.jl:48-55, test/Mana_test.jl:1-12) and Julia is absent here, so the
 * numeric functions are pinned only to analytic known answers and to the naive
 * O(8^n) restatement: "parity unpinned" for SRE/Mana values in the strict sense.
 *
 * Every function cites the reference file:line it restates.  All indices follow
 * the reference's conventions (1-based where the reference is 1-based, noted).
 *
 * The fast Walsh-Hadamard transform used by the reference is the external C library
 * FFHT, pulled as FastHadamardStructuredTransforms_jll v0.0.1 (Project.toml:9,31;
 * called at src/Helpers.jl:46-55,90).  It is not vendored; or_fwht below is written
 * from the definition of the in-place unnormalised transform
 *     v[k] <- sum_r (-1)^{popcount(k&r)} v[r],
 * applied stage by stage as (a, b) -> (a + b, a - b), the convention the reference's
 * CUDA extension also uses (ext/HadaMAGCUDAExt.jl:85-90).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include <immintrin.h>

#define OR_OK 0
#define OR_ERR_ARG -1

/* ------------------------------------------------------------------------- */
/* Gray codes                                                                 */
/* ------------------------------------------------------------------------- */

/* src/Basis.jl:14-27 (generate_binary): codes[k] = k ^ (k >> 1) for k = 0..2^n-1,
 * flips[k] (k = 0..2^n-2) = 1-based position of the bit that flips between codes[k]
 * and codes[k+1]. */
int or_gray_binary(int n, uint64_t *codes, int64_t *flips) {
    if (n < 0 || n > 40) return OR_ERR_ARG;
    uint64_t N = (uint64_t)1 << n;
    for (uint64_t i = 0; i < N; i++) codes[i] = i ^ (i >> 1);
    for (uint64_t k = 0; k + 1 < N; k++) flips[k] = (int64_t)__builtin_ctzll(codes[k] ^ codes[k + 1]) + 1;
    return OR_OK;
}

/* src/Helpers.jl:18-23 (partition_counts): split n items into P parts, the first
 * (n mod P) parts one larger; displs are the exclusive prefix sums. */
void or_partition_counts(int64_t n, int P, int64_t *counts, int64_t *displs) {
    int64_t base = n / P, rem = n % P, acc = 0;
    for (int i = 0; i < P; i++) {
        counts[i] = (i < rem) ? base + 1 : base;
        displs[i] = acc;
        acc += counts[i];
    }
}

/* src/Basis.jl:76-106 (generate_binary_splitted): the Gray codes of rank's slice of
 * the partition_counts split and the 1-based flips internal to the slice. */
int or_gray_binary_split(int n, int rank, int P, uint64_t *codes, int64_t *flips, int64_t *code_off) {
    if (n < 0 || n > 40 || P < 1 || rank < 0 || rank >= P) return OR_ERR_ARG;
    int64_t *cnt = malloc(sizeof(int64_t) * P), *dsp = malloc(sizeof(int64_t) * P);
    or_partition_counts((int64_t)1 << n, P, cnt, dsp);
    int64_t off = dsp[rank], c = cnt[rank];
    for (int64_t j = 0; j < c; j++) {
        uint64_t i = (uint64_t)(off + j);
        codes[j] = i ^ (i >> 1);
    }
    for (int64_t j = 0; j + 1 < c; j++) flips[j] = (int64_t)__builtin_ctzll(codes[j] ^ codes[j + 1]) + 1;
    *code_off = off;
    free(cnt);
    free(dsp);
    return OR_OK;
}

/* src/Basis.jl:123-133 (integer_to_gray): base-q digits of val least-significant
 * first, padded to n, folded from the most significant digit down with a running
 * shift: gray[i] = (digit[i] + shift) mod q; shift += q - gray[i]. */
static void integer_to_gray(int64_t val, int q, int n, int64_t *gray) {
    int64_t digit[64];
    for (int i = 0; i < n; i++) {
        digit[i] = val % q;
        val /= q;
    }
    int64_t shift = 0;
    for (int i = n - 1; i >= 0; i--) {
        gray[i] = (digit[i] + shift) % q;
        shift += q - gray[i];
    }
}

/* src/Basis.jl:146-164 (generate_general): XTAB is n x q^n, column-major (column k is
 * integer_to_gray(k)), flips[k] = 1-based first digit where columns k and k+1 differ. */
int or_gray_general(int n, int q, int64_t *xtab, int64_t *flips) {
    if (n < 0 || n > 40 || q < 2) return OR_ERR_ARG;
    int64_t N = 1;
    for (int i = 0; i < n; i++) N *= q;
    for (int64_t k = 0; k < N; k++) integer_to_gray(k, q, n, xtab + k * n);
    for (int64_t k = 0; k + 1 < N; k++) {
        int64_t pos = 0;
        for (int i = 0; i < n; i++)
            if (xtab[k * n + i] != xtab[(k + 1) * n + i]) {
                pos = i + 1;
                break;
            }
        flips[k] = pos;
    }
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* Walsh-Hadamard transform (from the definition; see header)                 */
/* ------------------------------------------------------------------------- */

/* AVX2 implementation (the Makefile compiles for x86-64-v3).  A vector holds 4
 * consecutive doubles: element stages 0 and 1 run inside the vector (a permute and a
 * signed fused multiply-add each), higher stages run across vectors, three at a time on
 * 8 vectors held in registers (radix 8). */

/* radix-8 butterflies on x[0..8): pairs at distances 1, 2, 4 */
static inline void r8(__m256d *x) {
    for (int d = 1; d < 8; d <<= 1)
        for (int i = 0; i < 8; i++)
            if (!(i & d)) {
                __m256d a = x[i], b = x[i + d];
                x[i] = _mm256_add_pd(a, b);
                x[i + d] = _mm256_sub_pd(a, b);
            }
}

/* radix-4 butterflies on x[0..4): pairs at distances 1, 2 */
static inline void r4(__m256d *x) {
    for (int d = 1; d < 4; d <<= 1)
        for (int i = 0; i < 4; i++)
            if (!(i & d)) {
                __m256d a = x[i], b = x[i + d];
                x[i] = _mm256_add_pd(a, b);
                x[i + d] = _mm256_sub_pd(a, b);
            }
}

/* element stages 0 and 1 inside one vector: (a0+a1, a0-a1, ...) then pairs at distance 2 */
static inline __m256d inv01(__m256d v) {
    const __m256d s0 = _mm256_setr_pd(1.0, -1.0, 1.0, -1.0), s1 = _mm256_setr_pd(1.0, 1.0, -1.0, -1.0);
    v = _mm256_fmadd_pd(v, s0, _mm256_permute_pd(v, 0x5));
    return _mm256_fmadd_pd(v, s1, _mm256_permute4x64_pd(v, 0x4e));
}

/* element stages [s0, B) of a contiguous block of 2^B doubles (s0 >= 2) */
static void block_stages(double *p, int B, int s0) {
    const int64_t nv = (int64_t)1 << (B - 2);
    int s = s0;
    for (; s + 3 <= B; s += 3) {
        const int64_t h = (int64_t)1 << (s - 2);
        for (int64_t i = 0; i < nv; i += 8 * h)
            for (int64_t j = i; j < i + h; j++) {
                __m256d x[8];
                for (int k = 0; k < 8; k++) x[k] = _mm256_load_pd(p + 4 * (j + k * h));
                r8(x);
                for (int k = 0; k < 8; k++) _mm256_store_pd(p + 4 * (j + k * h), x[k]);
            }
    }
    for (; s < B; s++) {
        const int64_t h = (int64_t)1 << (s - 2);
        for (int64_t i = 0; i < nv; i += 2 * h)
            for (int64_t j = i; j < i + h; j++) {
                __m256d a = _mm256_load_pd(p + 4 * j), b = _mm256_load_pd(p + 4 * (j + h));
                _mm256_store_pd(p + 4 * j, _mm256_add_pd(a, b));
                _mm256_store_pd(p + 4 * (j + h), _mm256_sub_pd(a, b));
            }
    }
}

/* full transform of a contiguous, 32-byte aligned block of 2^B doubles, 2 <= B */
static void fwht_block(double *p, int B) {
    const int64_t nv = (int64_t)1 << (B - 2);
    if (B >= 5) {
        for (int64_t i = 0; i < nv; i += 8) {
            __m256d x[8];
            for (int k = 0; k < 8; k++) x[k] = inv01(_mm256_load_pd(p + 4 * (i + k)));
            r8(x);
            for (int k = 0; k < 8; k++) _mm256_store_pd(p + 4 * (i + k), x[k]);
        }
        block_stages(p, B, 5);
    } else {
        for (int64_t i = 0; i < nv; i++) _mm256_store_pd(p + 4 * i, inv01(_mm256_load_pd(p + 4 * i)));
        block_stages(p, B, 2);
    }
}

/* row stages [0, H) of the 2^H x bs row-major matrix v, restricted to the W columns
 * [c, c + W) (W a multiple of 4): the high index bits of the vector */
static void col_stages(double *v, int64_t bs, int H, int64_t c, int W) {
    const int64_t rows = (int64_t)1 << H;
    int s = 0;
    for (; s + 3 <= H; s += 3) {
        const int64_t h = (int64_t)1 << s;
        for (int64_t i = 0; i < rows; i += 8 * h)
            for (int64_t j = i; j < i + h; j++)
                for (int w = 0; w < W; w += 4) {
                    __m256d x[8];
                    double *b = v + j * bs + c + w;
                    for (int k = 0; k < 8; k++) x[k] = _mm256_load_pd(b + k * h * bs);
                    r8(x);
                    for (int k = 0; k < 8; k++) _mm256_store_pd(b + k * h * bs, x[k]);
                }
    }
    if (s + 2 <= H) {
        const int64_t h = (int64_t)1 << s;
        for (int64_t i = 0; i < rows; i += 4 * h)
            for (int64_t j = i; j < i + h; j++)
                for (int w = 0; w < W; w += 4) {
                    __m256d x[4];
                    double *b = v + j * bs + c + w;
                    for (int k = 0; k < 4; k++) x[k] = _mm256_load_pd(b + k * h * bs);
                    r4(x);
                    for (int k = 0; k < 4; k++) _mm256_store_pd(b + k * h * bs, x[k]);
                }
        s += 2;
    }
    for (; s < H; s++) {
        const int64_t h = (int64_t)1 << s;
        for (int64_t i = 0; i < rows; i += 2 * h)
            for (int64_t j = i; j < i + h; j++)
                for (int w = 0; w < W; w += 4) {
                    double *b = v + j * bs + c + w;
                    __m256d a = _mm256_load_pd(b), d = _mm256_load_pd(b + h * bs);
                    _mm256_store_pd(b, _mm256_add_pd(a, d));
                    _mm256_store_pd(b + h * bs, _mm256_sub_pd(a, d));
                }
    }
}

/* Split of an L-bit transform: the low B bits on contiguous blocks of 2^B doubles (16 KiB,
 * L1-resident), then the high L-B bits on column blocks of W doubles x 2^(L-B) rows
 * (L2-resident): two sweeps over the vector in all. */
#define OR_FWHT_LOW_BITS 11
#define OR_FWHT_COLS 128

/* 64-byte aligned buffer of `count` doubles (at least 8) */
static double *or_valloc(int64_t count) {
    size_t bytes = sizeof(double) * (size_t)(count < 8 ? 8 : count);
    bytes = (bytes + 63) & ~(size_t)63;
    return aligned_alloc(64, bytes);
}

static void fwht_small(double *v, int L) { /* L < 2: plain butterflies */
    if (L == 1) {
        double a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
}

/* in-place unnormalised WHT of v[0 .. 2^L); v 32-byte aligned when L >= 2 */
void or_fwht(double *v, int L) {
    if (L <= 1) {
        fwht_small(v, L);
        return;
    }
    if (((uintptr_t)v & 31) != 0) { /* unaligned caller buffer: transform an aligned copy */
        const size_t bytes = sizeof(double) * ((size_t)1 << L);
        double *a = or_valloc((int64_t)1 << L);
        memcpy(a, v, bytes);
        or_fwht(a, L);
        memcpy(v, a, bytes);
        free(a);
        return;
    }
    const int64_t N = (int64_t)1 << L;
    const int B = L < OR_FWHT_LOW_BITS ? L : OR_FWHT_LOW_BITS;
    const int64_t bs = (int64_t)1 << B;
    for (int64_t base = 0; base < N; base += bs) fwht_block(v + base, B);
    if (L > B)
        for (int64_t c = 0; c < bs; c += OR_FWHT_COLS) col_stages(v, bs, L - B, c, OR_FWHT_COLS);
}

/* ------------------------------------------------------------------------- */
/* Exact SRE                                                                  */
/* ------------------------------------------------------------------------- */

/* (F^2)^q for the reference's two cases: q == 2 -> p*p (src/SRE.jl:239), other q ->
 * p^q (src/SRE.jl:262; integer q by repeated product, non-integer by pow). */
static inline double pow_q(double p, double q) {
    if (q == 2.0) return p * p;
    if (q == floor(q) && q >= 1.0 && q <= 16.0) {
        double r = p;
        for (int i = 1; i < (int)q; i++) r *= p;
        return r;
    }
    return pow(p, q);
}

/* src/SRE.jl:225-278 (kahan_accumulate): per-x compensated sums of p = v^2 and of
 * (p)^q over the transformed vector. */
static void kahan_accumulate(const double *restrict v, int64_t dim, double q, double *p2_out, double *m_out) {
    double p2_sum = 0.0, p2_c = 0.0, m_sum = 0.0, m_c = 0.0;
    for (int64_t i = 0; i < dim; i++) {
        double p = v[i] * v[i];
        double pq = pow_q(p, q);
        double y = p - p2_c;
        double t = p2_sum + y;
        p2_c = (t - p2_sum) - y;
        p2_sum = t;
        double y2 = pq - m_c;
        double t2 = m_sum + y2;
        m_c = (t2 - m_sum) - y2;
        m_sum = t2;
    }
    *p2_out = p2_sum;
    *m_out = m_sum;
}

/* src/SRE.jl:509-540 (flip_and_update_mask!): inVR[r] = X1[r]*TMP1[r^mask] +
 * X2[r]*TMP2[r^mask] with mask = old mask ^ (1 << site); written as the reference's
 * muladd(X1, TMP1[j], X2 * TMP2[j]).  Returns the new mask. */
static uint64_t flip_and_update_mask(int site, int64_t dim, uint64_t mask, const double *TMP1, const double *TMP2,
                                     const double *X1, const double *X2, double *inVR) {
    uint64_t newmask = mask ^ ((uint64_t)1 << site);
    for (int64_t r = 0; r < dim; r++) {
        uint64_t j = (uint64_t)r ^ newmask;
        inVR[r] = fma(X1[r], TMP1[j], X2[r] * TMP2[j]);
    }
    return newmask;
}

typedef struct {
    int n;
    int64_t dim;
    double *X1, *X2, *TMP1, *TMP2; /* src/Backends/Threads.jl:115-128 */
} sre_prep;

static int sre_prep_init(sre_prep *s, const double *psi, int n) {
    s->n = n;
    s->dim = (int64_t)1 << n;
    size_t bytes = sizeof(double) * (size_t)s->dim;
    s->X1 = malloc(bytes);
    s->X2 = malloc(bytes);
    s->TMP1 = malloc(bytes);
    s->TMP2 = malloc(bytes);
    if (!s->X1 || !s->X2 || !s->TMP1 || !s->TMP2) return OR_ERR_ARG;
    for (int64_t i = 0; i < s->dim; i++) {
        double r = psi[2 * i], im = psi[2 * i + 1];
        s->X1[i] = r;
        s->X2[i] = im;
        s->TMP1[i] = r + im;
        s->TMP2[i] = im - r;
    }
    return OR_OK;
}

static void sre_prep_free(sre_prep *s) {
    free(s->X1);
    free(s->X2);
    free(s->TMP1);
    free(s->TMP2);
}

/* src/SRE.jl:338-411 and 424-496 (compute_chunk_sre): Gray walk over 1-based Gray
 * indices ix = istart..iend.  At the chunk head the mask is rebuilt from all set bits of
 * XTAB[istart] (or one plain blend when it is 0); afterwards one site flips per step.
 * Per x: blend, FWHT, Kahan sums; the chunk totals p2SAM, mSAM are plain sums. */
static void sre_chunk(const sre_prep *s, double q, int64_t istart, int64_t iend, double *inVR, double *p2_out,
                      double *m_out) {
    const int64_t dim = s->dim;
    double p2SAM = 0.0, mSAM = 0.0;
    uint64_t mask = 0;
    for (int64_t ix = istart; ix <= iend; ix++) {
        if (ix == istart) {
            uint64_t k = (uint64_t)(ix - 1);
            uint64_t bits = k ^ (k >> 1); /* XTAB[ix] */
            if (bits == 0) {
                for (int64_t r = 0; r < dim; r++) inVR[r] = fma(s->X1[r], s->TMP1[r], s->X2[r] * s->TMP2[r]);
            } else {
                uint64_t m = bits;
                while (m != 0) {
                    int site = __builtin_ctzll(m);
                    mask = flip_and_update_mask(site, dim, mask, s->TMP1, s->TMP2, s->X1, s->X2, inVR);
                    m &= m - 1;
                }
            }
        } else {
            /* Zwhere[ix-1] - 1: 0-based site flipping between XTAB[ix-1] and XTAB[ix] */
            uint64_t a = (uint64_t)(ix - 2), b = (uint64_t)(ix - 1);
            int site = __builtin_ctzll((a ^ (a >> 1)) ^ (b ^ (b >> 1)));
            mask = flip_and_update_mask(site, dim, mask, s->TMP1, s->TMP2, s->X1, s->X2, inVR);
        }
        or_fwht(inVR, s->n);
        double lp2, lm;
        kahan_accumulate(inVR, dim, q, &lp2, &lm);
        p2SAM += lp2;
        mSAM += lm;
    }
    *p2_out = p2SAM;
    *m_out = mSAM;
}

/* Raw sums (p2SAM, mSAM) over 1-based Gray indices [istart, iend] split over nthreads
 * exactly as src/Backends/Threads.jl:37-102 (threaded_chunk_reduce): static contiguous
 * partition_counts slices, per-thread compute_chunk_sre, per-thread results summed in
 * thread order. */
int or_sre_sums(const double *psi, int n, double q, int64_t istart, int64_t iend, int nthreads, double *p2_out,
                double *m_out) {
    if (n < 0 || n > 30 || nthreads < 1) return OR_ERR_ARG;
    const int64_t dim = (int64_t)1 << n;
    if (istart < 1 || iend > dim || iend < istart - 1) return OR_ERR_ARG;
    sre_prep s;
    if (sre_prep_init(&s, psi, n) != OR_OK) return OR_ERR_ARG;
    const int64_t len = iend - istart + 1;
    int64_t *tcnt = malloc(sizeof(int64_t) * nthreads), *tdisp = malloc(sizeof(int64_t) * nthreads);
    double *acc = calloc(2 * (size_t)nthreads, sizeof(double));
    or_partition_counts(len, nthreads, tcnt, tdisp);
#pragma omp parallel num_threads(nthreads)
    {
        int tid = omp_get_thread_num();
        if (tid < nthreads && tcnt[tid] > 0) {
            double *inVR = or_valloc(dim);
            int64_t a = istart + tdisp[tid], b = istart + tdisp[tid] + tcnt[tid] - 1;
            sre_chunk(&s, q, a, b, inVR, &acc[2 * tid], &acc[2 * tid + 1]);
            free(inVR);
        }
    }
    double p2 = 0.0, m = 0.0;
    for (int t = 0; t < nthreads; t++) {
        p2 += acc[2 * t];
        m += acc[2 * t + 1];
    }
    *p2_out = p2;
    *m_out = m;
    free(tcnt);
    free(tdisp);
    free(acc);
    sre_prep_free(&s);
    return OR_OK;
}

/* double-double accumulation (Knuth TwoSum) for the fast path's cross-X-string sums */
static inline void dd_acc(double *hi, double *lo, double b) {
    double s = *hi + b, bb = s - *hi;
    *lo += (*hi - (s - bb)) + (b - bb);
    *hi = s;
}

/* sums of y = v^2 and y^2 (and y^3 when q3) over count doubles of p, 4-lane FP64 */
static void moments23(const double *p, int64_t count, int q3, double *t2, double *t4, double *t6) {
    __m256d a2 = _mm256_setzero_pd(), a4 = a2, a6 = a2, b2 = a2, b4 = a2, b6 = a2;
    int64_t e = 0;
    for (; e + 8 <= count; e += 8) {
        __m256d v = _mm256_loadu_pd(p + e), w = _mm256_loadu_pd(p + e + 4);
        __m256d y = _mm256_mul_pd(v, v), z = _mm256_mul_pd(w, w);
        a2 = _mm256_add_pd(a2, y);
        b2 = _mm256_add_pd(b2, z);
        a4 = _mm256_fmadd_pd(y, y, a4);
        b4 = _mm256_fmadd_pd(z, z, b4);
        if (q3) {
            a6 = _mm256_fmadd_pd(_mm256_mul_pd(y, y), y, a6);
            b6 = _mm256_fmadd_pd(_mm256_mul_pd(z, z), z, b6);
        }
    }
    double l2[4], l4[4], l6[4];
    _mm256_storeu_pd(l2, _mm256_add_pd(a2, b2));
    _mm256_storeu_pd(l4, _mm256_add_pd(a4, b4));
    _mm256_storeu_pd(l6, _mm256_add_pd(a6, b6));
    double s2 = (l2[0] + l2[1]) + (l2[2] + l2[3]), s4 = (l4[0] + l4[1]) + (l4[2] + l4[3]);
    double s6 = (l6[0] + l6[1]) + (l6[2] + l6[3]);
    for (; e < count; e++) {
        const double y = p[e] * p[e];
        s2 += y;
        s4 += y * y;
        s6 += y * y * y;
    }
    *t2 = s2;
    *t4 = s4;
    *t6 = s6;
}

/* v[r] = muladd(X1[r], TMP1[r^x], X2[r] TMP2[r^x]) for r in [base, base + bs), bs >= 4:
 * vector loads at (r ^ x) with the low two bits of x applied as a lane permutation */
static inline __m256d perm_lanes(__m256d a, int m) {
    switch (m) {
        case 1: return _mm256_permute_pd(a, 0x5);
        case 2: return _mm256_permute4x64_pd(a, 0x4e);
        case 3: return _mm256_permute4x64_pd(a, 0x1b);
        default: return a;
    }
}
static void build_block(const sre_prep *s, uint64_t x, int64_t base, int64_t bs, double *v) {
    const int m = (int)(x & 3);
    const uint64_t xv = x & ~(uint64_t)3;
    for (int64_t r = base; r < base + bs; r += 4) {
        const uint64_t j = (uint64_t)r ^ xv;
        const __m256d t1 = perm_lanes(_mm256_loadu_pd(s->TMP1 + j), m);
        const __m256d t2 = perm_lanes(_mm256_loadu_pd(s->TMP2 + j), m);
        const __m256d x1 = _mm256_loadu_pd(s->X1 + r), x2 = _mm256_loadu_pd(s->X2 + r);
        _mm256_storeu_pd(v + r, _mm256_fmadd_pd(x1, t1, _mm256_mul_pd(x2, t2)));
    }
}

/* One thread's share of the fast path: 1-based Gray indices [ia, ib], double-double
 * sums into a[2 (1 + nq)] (added to what a holds). */
static void sre_fast_span(const sre_prep *s, const double *qs, int nq, int64_t ia, int64_t ib, double *a) {
    const int n = s->n;
    const int64_t dim = s->dim;
    int only23 = 1, has3 = 0;
    for (int qi = 0; qi < nq; qi++) {
        if (qs[qi] != 2.0 && qs[qi] != 3.0) only23 = 0;
        if (qs[qi] == 3.0) has3 = 1;
    }
    const int B = n < OR_FWHT_LOW_BITS ? n : OR_FWHT_LOW_BITS, H = n - B;
    const int64_t bs = (int64_t)1 << B, rows = (int64_t)1 << H;
    const int W = bs < OR_FWHT_COLS ? (int)bs : OR_FWHT_COLS;
    double *v = or_valloc(dim);
    double *col = or_valloc(rows * W);
    for (int64_t ix = ia; ix <= ib; ix++) {
        const uint64_t k = (uint64_t)(ix - 1), x = k ^ (k >> 1);
        for (int64_t base = 0; base < dim; base += bs) {
            build_block(s, x, base, bs, v);
            fwht_block(v + base, B);
        }
        double xs[5][2] = {{0}};
        for (int64_t c = 0; c < bs; c += W) {
            if (H > 0) col_stages(v, bs, H, c, W);
            /* gather the column block contiguously for the moment sums */
            for (int64_t r = 0; r < rows; r++) memcpy(col + r * W, v + r * bs + c, sizeof(double) * W);
            double t[5] = {0};
            if (only23) {
                double t2, t4, t6;
                moments23(col, rows * W, has3, &t2, &t4, &t6);
                t[0] = t2;
                for (int qi = 0; qi < nq; qi++) t[1 + qi] = qs[qi] == 2.0 ? t4 : t6;
            } else {
                for (int64_t e = 0; e < rows * W; e++) {
                    const double y = col[e] * col[e];
                    t[0] += y;
                    for (int qi = 0; qi < nq; qi++) t[1 + qi] += pow_q(y, qs[qi]);
                }
            }
            for (int u = 0; u <= nq; u++) dd_acc(&xs[u][0], &xs[u][1], t[u]);
        }
        for (int u = 0; u <= nq; u++) {
            dd_acc(&a[2 * u], &a[2 * u + 1], xs[u][0]);
            a[2 * u + 1] += xs[u][1];
        }
    }
    free(col);
    free(v);
}

/* Fast path of or_sre_sums, several q per transform: the same Gray walk split, build
 * (src/SRE.jl:509-540, inVR[r] = muladd(X1[r], TMP1[r^x], X2[r] TMP2[r^x]) computed
 * straight from x, as flip_and_update_mask recomputes every entry anyway), FWHT and
 * moments, with the build fused into the transform's low-bit sweep and the moments into
 * its high-bit sweep, so the vector crosses memory twice per X-string.  The per-x
 * moments are summed per column block (plain FP64 in 8 lanes) and the block sums in
 * double-double, as are the sums across X-strings and threads; the reference's
 * @fastmath Kahan loop (src/SRE.jl:225-278) defines no finer order.  Used for the large
 * fixtures and the timed CPU baseline; parity tests at small n use or_sre_sums.
 * Thread t takes the t-th contiguous partition_counts slice of [istart, iend]
 * (src/Backends/Threads.jl:37-102); with per_thread > 0 it takes only the first
 * per_thread indices of its slice, which is how a :threads run starts (the timed
 * sample of the CPU baseline).
 * out: 2 (1 + nq) doubles, (hi, lo) of sum F^2 then of sum (F^2)^q per q. */
int or_sre_sums_fast(const double *psi, int n, const double *qs, int nq, int64_t istart, int64_t iend,
                     int64_t per_thread, int nthreads, double *out) {
    if (n < 2 || n > 30 || nthreads < 1 || nq < 1 || nq > 4) return OR_ERR_ARG;
    const int64_t dim = (int64_t)1 << n;
    if (istart < 1 || iend > dim || iend < istart - 1) return OR_ERR_ARG;
    sre_prep s;
    if (sre_prep_init(&s, psi, n) != OR_OK) return OR_ERR_ARG;
    const int64_t len = iend - istart + 1;
    int64_t *tcnt = malloc(sizeof(int64_t) * nthreads), *tdisp = malloc(sizeof(int64_t) * nthreads);
    double *acc = calloc(2 * 5 * (size_t)nthreads, sizeof(double));
    or_partition_counts(len, nthreads, tcnt, tdisp);
#pragma omp parallel num_threads(nthreads)
    {
        int tid = omp_get_thread_num();
        if (tid < nthreads && tcnt[tid] > 0) {
            int64_t cnt = tcnt[tid];
            if (per_thread > 0 && per_thread < cnt) cnt = per_thread;
            sre_fast_span(&s, qs, nq, istart + tdisp[tid], istart + tdisp[tid] + cnt - 1, acc + 10 * (size_t)tid);
        }
    }
    for (int u = 0; u < 2 * (1 + nq); u++) out[u] = 0.0;
    for (int t = 0; t < nthreads; t++)
        for (int u = 0; u <= nq; u++) {
            dd_acc(&out[2 * u], &out[2 * u + 1], acc[10 * t + 2 * u]);
            out[2 * u + 1] += acc[10 * t + 2 * u + 1];
        }
    free(tcnt);
    free(tdisp);
    free(acc);
    sre_prep_free(&s);
    return OR_OK;
}

/* src/Backends/Threads.jl:108-159 (SRE): (-log2(m/dim), |1 - p2/dim|) over all 2^n
 * X-strings.  With nthreads == 1 this is src/Backends/Serial.jl:7-51. */
int or_sre(const double *psi, int n, double q, int nthreads, double *sre, double *lost) {
    double p2, m;
    const int64_t dim = (int64_t)1 << n;
    int rc = or_sre_sums(psi, n, q, 1, dim, nthreads, &p2, &m);
    if (rc != OR_OK) return rc;
    *sre = -log2(m / (double)dim);
    *lost = fabs(1.0 - p2 / (double)dim);
    return OR_OK;
}

/* src/SRE.jl:601-679 (iphase, expval_pauli_mask): <psi|P_{x,z}|psi> =
 * real(i^{|x&z|} * sum_b (-1)^{b.z} conj(psi[b^x]) psi[b]). */
static double expval_pauli_mask(const double *psi, int64_t N, uint64_t x, uint64_t z) {
    int k = __builtin_popcountll(x & z) & 3;
    double sr = 0.0, si = 0.0;
    for (int64_t b = 0; b < N; b++) {
        uint64_t bp = (uint64_t)b ^ x;
        double sign = (__builtin_popcountll((uint64_t)b & z) & 1) ? -1.0 : 1.0;
        double ar = psi[2 * bp], ai = -psi[2 * bp + 1]; /* conj(psi[b^x]) */
        double br = psi[2 * b], bi = psi[2 * b + 1];
        sr += sign * (ar * br - ai * bi);
        si += sign * (ar * bi + ai * br);
    }
    /* real(i^k * (sr + i si)) */
    switch (k) {
        case 0: return sr;
        case 1: return -si;
        case 2: return -sr;
        default: return si;
    }
}

/* src/SRE.jl:690-749 (naive_SRE): -log2( sum over all 4^n Pauli strings of
 * (e^2)^q / N ) with per-thread compensated sums, the Pauli string decoded from the
 * base-4 digits of idx (0 -> I, 1 -> X, 2 -> Y, 3 -> Z). */
int or_naive_sre(const double *psi, int n, int q, int nthreads, double *out) {
    if (n < 0 || n > 14 || q < 1 || nthreads < 1) return OR_ERR_ARG;
    const int64_t N = (int64_t)1 << n;
    const int64_t total = (int64_t)1 << (2 * n);
    double *partial = calloc((size_t)nthreads, sizeof(double));
    double *cval = calloc((size_t)nthreads, sizeof(double));
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t idx = 0; idx < total; idx++) {
        int tid = omp_get_thread_num();
        uint64_t tmp = (uint64_t)idx, x = 0, z = 0;
        for (int j = 0; j < n; j++) {
            uint64_t d = tmp & 3;
            if (d == 1) x |= (uint64_t)1 << j;
            else if (d == 2) { x |= (uint64_t)1 << j; z |= (uint64_t)1 << j; }
            else if (d == 3) z |= (uint64_t)1 << j;
            tmp >>= 2;
        }
        double e = expval_pauli_mask(psi, N, x, z);
        double p = e * e, pq = p;
        for (int i = 1; i < q; i++) pq *= p;
        double y = pq - cval[tid];
        double t = partial[tid] + y;
        cval[tid] = (t - partial[tid]) - y;
        partial[tid] = t;
    }
    double s = 0.0;
    for (int t = 0; t < nthreads; t++) s += partial[t];
    *out = -log2(s / (double)N);
    free(partial);
    free(cval);
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* Monte-Carlo SRE (Metropolis over X-strings)                                */
/* ------------------------------------------------------------------------- */

/* src/SRE.jl:195-223 (compute_moments): plain sums of v^2 and of (v^2)^q. */
static void compute_moments(const double *v, int64_t dim, double q, double *s2, double *s4) {
    double a = 0.0, b = 0.0;
    for (int64_t i = 0; i < dim; i++) {
        double y2 = v[i] * v[i];
        a += y2;
        if (q == 2.0) b = fma(y2, y2, b);
        else b += pow_q(y2, q);
    }
    *s2 = a;
    *s4 = b;
}

/* src/SRE.jl:127-140 (blend_mask!, sample_mask!): inVR[i] = muladd(re X[i],
 * tmp1[i^mask], im X[i] * tmp2[i^mask]), FWHT, moments; returns (p2/dim, m_q). */
static void sample_mask(const sre_prep *s, double q, uint64_t mask, double *inVR, double *p2, double *mq) {
    for (int64_t i = 0; i < s->dim; i++) {
        uint64_t j = (uint64_t)i ^ mask;
        inVR[i] = fma(s->X1[i], s->TMP1[j], s->X2[i] * s->TMP2[j]);
    }
    or_fwht(inVR, s->n);
    double a, b;
    compute_moments(inVR, s->dim, q, &a, &b);
    *p2 = a / (double)s->dim;
    *mq = b;
}

/* src/SRE.jl:110-192 (mc_sre_beta!) with the proposal stream injected: the reference
 * draws tries[t] = floor(9 u) + 1 site flips, each site = rand(rng, 1:L), and
 * propDelta[t] = XOR of those site bits, plus rs[t] uniform in [0,1)
 * (src/SRE.jl:142-145,164-170).  Those draws are inputs here (prop_delta, rs).
 * out5 = (mean M2, mean M2^2, m0/dim, mean P2, n); accepted (optional, nsamples)
 * records the current mask after each step. */
int or_mc_sre_beta(const double *psi, int n, double q, int nsamples, double beta, const uint64_t *prop_delta,
                   const double *rs, double *out5, uint64_t *masks_out) {
    if (n < 0 || n > 30 || nsamples < 1) return OR_ERR_ARG;
    sre_prep s;
    if (sre_prep_init(&s, psi, n) != OR_OK) return OR_ERR_ARG;
    double *inVR = malloc(sizeof(double) * (size_t)s.dim);
    double p2_0, m0;
    sample_mask(&s, q, 0, inVR, &p2_0, &m0);
    uint64_t currMask = 0;
    double currPROB = 1e-120, currM2 = 0.0, currP2 = p2_0;
    double sM2 = 0.0, sM2sq = 0.0, sP2 = 0.0;
    int64_t cnt = 0;
    for (int t = 0; t < nsamples; t++) {
        uint64_t propMask = currMask ^ prop_delta[t];
        double p2_prop, m_prop;
        sample_mask(&s, q, propMask, inVR, &p2_prop, &m_prop);
        double pb = pow(m_prop, beta);
        double r = rs[t];
        if ((r < pb / currPROB) && (propMask != 0)) {
            currMask = propMask;
            currPROB = pb;
            currM2 = -log2(m_prop);
            currP2 = p2_prop;
        }
        sM2 += currM2;
        sM2sq += currM2 * currM2;
        sP2 += currP2;
        cnt += 1;
        if (masks_out) masks_out[t] = currMask;
    }
    out5[0] = sM2 / (double)cnt;
    out5[1] = sM2sq / (double)cnt;
    out5[2] = m0 / (double)s.dim;
    out5[3] = sP2 / (double)cnt;
    out5[4] = (double)cnt;
    free(inVR);
    sre_prep_free(&s);
    return OR_OK;
}

/* src/Helpers.jl:223-236 (integrate_simpson_uniform). */
double or_simpson_uniform(const double *x, const double *y, int npts) {
    int n = npts - 1;
    if (n <= 0 || n % 2 != 0) return NAN;
    double h = (x[npts - 1] - x[0]) / n;
    double odd = 0.0, even = 0.0;
    for (int i = 1; i < npts - 1; i += 2) odd += y[i];
    for (int i = 2; i < npts - 1; i += 2) even += y[i];
    return (h / 3.0) * (y[0] + y[npts - 1] + 4.0 * odd + 2.0 * even);
}

/* src/Backends/Threads.jl:161-221 (MC_SRE): one chain per beta_i = (i-1)/(Nbeta-1),
 * Simpson over M2 and M2ADD, m2 = -log2(2^-I + I_add).  prop_delta and rs hold
 * Nbeta consecutive streams of nsamples each. */
int or_mc_sre(const double *psi, int n, double q, int nbeta, int nsamples, const uint64_t *prop_delta,
              const double *rs, int nthreads, double *m2_out, double *M2, double *M2ADD, double *P2) {
    if (nbeta < 3 || nbeta % 2 != 1) return OR_ERR_ARG;
    int rc = OR_OK;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < nbeta; i++) {
        double beta = (double)i / (double)(nbeta - 1);
        double o[5];
        int r = or_mc_sre_beta(psi, n, q, nsamples, beta, prop_delta + (size_t)i * nsamples,
                               rs + (size_t)i * nsamples, o, NULL);
        if (r != OR_OK) rc = r;
        M2[i] = o[0];
        M2ADD[i] = o[2];
        P2[i] = o[3];
    }
    if (rc != OR_OK) return rc;
    double *x = malloc(sizeof(double) * nbeta);
    for (int i = 0; i < nbeta; i++) x[i] = (double)i / (double)(nbeta - 1);
    double I_res = or_simpson_uniform(x, M2, nbeta);
    double I_add = or_simpson_uniform(x, M2ADD, nbeta);
    *m2_out = -log2(pow(2.0, -I_res) + I_add);
    free(x);
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* Mana (qutrits)                                                             */
/* ------------------------------------------------------------------------- */

/* src/Helpers.jl:246-292 (fast_hadamard_qutrit!): L stages of the 3-point DFT
 * (a, b, c) -> (a+b+c, a+w b+w^2 c, a+w^2 b+w c), w = e^{2 pi i/3}, on interleaved
 * complex data of length N = 3^L. */
void or_fht_qutrit(double *v, int64_t N) {
    const double wr = -0.5, wi = sqrt(3.0) / 2.0;
    int64_t step = 1;
    while (step < N) {
        int64_t jump = 3 * step;
        for (int64_t i = 0; i < N; i += jump)
            for (int64_t j = 0; j < step; j++) {
                int64_t ia = i + j, ib = ia + step, ic = ia + 2 * step;
                double ar = v[2 * ia], ai = v[2 * ia + 1];
                double br = v[2 * ib], bi = v[2 * ib + 1];
                double cr = v[2 * ic], ci = v[2 * ic + 1];
                double r0 = ar + br + cr, i0 = ai + bi + ci;
                double r1 = ar + wr * (br + cr) - wi * (bi - ci);
                double i1 = ai + wr * (bi + ci) + wi * (br - cr);
                double r2 = ar + wr * (br + cr) + wi * (bi - ci);
                double i2 = ai + wr * (bi + ci) - wi * (br - cr);
                v[2 * ia] = r0; v[2 * ia + 1] = i0;
                v[2 * ib] = r1; v[2 * ib + 1] = i1;
                v[2 * ic] = r2; v[2 * ic + 1] = i2;
            }
        step = jump;
    }
}

/* src/Mana.jl:97-113 (rotate_perm_site!): cyclic update of the permutation for the
 * qutrit shift at 1-based site, k = 1 (0->1->2) or k = 2 (0->2->1). */
static void rotate_perm_site(int64_t *perm, int64_t len, int site, int k) {
    int64_t stride = 1;
    for (int i = 1; i < site; i++) stride *= 3;
    int64_t block = 3 * stride;
    for (int64_t bs = 0; bs < len; bs += block)
        for (int64_t off = 0; off < stride; off++) {
            int64_t i0 = bs + off, i1 = i0 + stride, i2 = i1 + stride;
            int64_t p0 = perm[i0], p1 = perm[i1], p2 = perm[i2];
            if (k == 1) { perm[i0] = p1; perm[i1] = p2; perm[i2] = p0; }
            else { perm[i0] = p2; perm[i1] = p0; perm[i2] = p1; }
        }
}

/* src/Mana.jl:19-92 (compute_chunk_mana_qutrits): columns ix = istart..iend (1-based)
 * of the ternary Gray table; per column inV[r] = conj(psi[perm[r]]) * (psi[perm[AA[r]]]
 * / 3^L), qutrit Hadamard, running Kahan sum of |inV| across the chunk; the
 * permutation advances by one single-site rotation per column. */
static double mana_chunk(const double *psi, int L, int64_t dim, const int64_t *XTAB, const int64_t *Zwhere,
                         const int64_t *AA, int64_t istart, int64_t iend, double *inV) {
    const double invdim = 1.0 / (double)dim;
    int64_t *perm = malloc(sizeof(int64_t) * (size_t)dim);
    for (int64_t i = 0; i < dim; i++) perm[i] = i;
    for (int s = 1; s <= L; s++) {
        int64_t k = XTAB[(istart - 1) * L + (s - 1)] % 3;
        if (k == 1) rotate_perm_site(perm, dim, s, 1);
        else if (k == 2) rotate_perm_site(perm, dim, s, 2);
    }
    double p2SAM = 0.0, c = 0.0;
    for (int64_t ix = istart; ix <= iend; ix++) {
        for (int64_t r = 0; r < dim; r++) {
            int64_t pa = perm[r], pb = perm[AA[r]];
            double ar = psi[2 * pa], ai = psi[2 * pa + 1];
            double br = psi[2 * pb] * invdim, bi = psi[2 * pb + 1] * invdim;
            /* conj(a) * b */
            inV[2 * r] = ar * br + ai * bi;
            inV[2 * r + 1] = ar * bi - ai * br;
        }
        or_fht_qutrit(inV, dim);
        for (int64_t i = 0; i < dim; i++) {
            double ap = hypot(inV[2 * i], inV[2 * i + 1]);
            double y = ap - c;
            double t = p2SAM + y;
            c = (t - p2SAM) - y;
            p2SAM = t;
        }
        if (ix < iend) {
            int s = (int)Zwhere[ix - 1];
            int64_t kstep = ((XTAB[ix * L + (s - 1)] - XTAB[(ix - 1) * L + (s - 1)]) % 3 + 3) % 3;
            rotate_perm_site(perm, dim, s, (int)kstep);
        }
    }
    free(perm);
    return p2SAM;
}

/* Sum of |W| over the 1-based ternary Gray columns [istart, iend], threaded as
 * src/Backends/Threads.jl:223-271 (static partition, thread-ordered sum). */
int or_mana_sum(const double *psi, int L, int64_t istart, int64_t iend, int nthreads, double *sum_out) {
    if (L < 0 || L > 16 || nthreads < 1) return OR_ERR_ARG;
    int64_t dim = 1;
    for (int i = 0; i < L; i++) dim *= 3;
    if (istart < 1 || iend > dim || iend < istart) return OR_ERR_ARG;
    int64_t *XTAB = malloc(sizeof(int64_t) * (size_t)dim * (L > 0 ? L : 1));
    int64_t *Zwhere = malloc(sizeof(int64_t) * (size_t)dim);
    or_gray_general(L, 3, XTAB, Zwhere);
    /* src/Backends/Threads.jl:229-242: AA = digitwise negation mod 3 (0-based here) */
    int64_t *AA = malloc(sizeof(int64_t) * (size_t)dim);
    for (int64_t i = 0; i < dim; i++) {
        int64_t x = i, y = 0, pw = 1;
        for (int k = 0; k < L; k++) {
            int64_t d = x % 3;
            x /= 3;
            y += ((3 - d) % 3) * pw;
            pw *= 3;
        }
        AA[i] = y;
    }
    const int64_t len = iend - istart + 1;
    int64_t *tcnt = malloc(sizeof(int64_t) * nthreads), *tdisp = malloc(sizeof(int64_t) * nthreads);
    double *acc = calloc((size_t)nthreads, sizeof(double));
    or_partition_counts(len, nthreads, tcnt, tdisp);
#pragma omp parallel num_threads(nthreads)
    {
        int tid = omp_get_thread_num();
        if (tcnt[tid] > 0) {
            double *inV = malloc(sizeof(double) * 2 * (size_t)dim);
            acc[tid] = mana_chunk(psi, L, dim, XTAB, Zwhere, AA, istart + tdisp[tid],
                                  istart + tdisp[tid] + tcnt[tid] - 1, inV);
            free(inV);
        }
    }
    double s = 0.0;
    for (int t = 0; t < nthreads; t++) s += acc[t];
    *sum_out = s;
    free(XTAB);
    free(Zwhere);
    free(AA);
    free(tcnt);
    free(tdisp);
    free(acc);
    return OR_OK;
}

/* src/Backends/Threads.jl:223-271 (Mana): log2(S)/log2(3). */
int or_mana_pure(const double *psi, int L, int nthreads, double *mana) {
    int64_t dim = 1;
    for (int i = 0; i < L; i++) dim *= 3;
    double s;
    int rc = or_mana_sum(psi, L, 1, dim, nthreads, &s);
    if (rc != OR_OK) return rc;
    *mana = log2(s) / log2(3.0);
    return OR_OK;
}

/* complex helpers (interleaved) */
typedef struct { double re, im; } cplx;
static inline cplx cmul(cplx a, cplx b) { cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cplx cadd(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cplx cconj(cplx a) { cplx r = {a.re, -a.im}; return r; }

static void mat3_mul(const cplx *A, const cplx *B, cplx *C) { /* row-major 3x3 */
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            cplx s = {0, 0};
            for (int k = 0; k < 3; k++) s = cadd(s, cmul(A[3 * i + k], B[3 * k + j]));
            C[3 * i + j] = s;
        }
}

/* src/Mana.jl:123-182 (build_single_qutrit_M): M is 9x9, row idx = vec_colmajor(A_u^T),
 * A_u = T_u A0 T_u^dagger, T_{a,a'} = w^{(-2 a a') mod 3} Z^a X^{a'}, idx = 3a + a',
 * A0 = (1/3) sum_u T_u.  Output M row-major: M[9*idx + c]. */
void or_single_qutrit_M(double *Mout) {
    const double PI = 3.14159265358979323846;
    cplx w = {cos(2 * PI / 3), sin(2 * PI / 3)};
    cplx X[9] = {{0}}, Z[9] = {{0}}, I3[9] = {{0}};
    for (int k = 0; k < 3; k++) {
        X[3 * ((k + 1) % 3) + k].re = 1.0; /* X[(k+1)%3, k] = 1 */
        I3[3 * k + k].re = 1.0;
    }
    cplx wp[3] = {{1, 0}, w, cmul(w, w)};
    for (int k = 0; k < 3; k++) Z[3 * k + k] = wp[k]; /* w^k */
    cplx Zp[3][9], Xp[3][9];
    memcpy(Zp[0], I3, sizeof(I3));
    memcpy(Zp[1], Z, sizeof(Z));
    mat3_mul(Z, Z, Zp[2]);
    memcpy(Xp[0], I3, sizeof(I3));
    memcpy(Xp[1], X, sizeof(X));
    mat3_mul(X, X, Xp[2]);
    cplx T[9][9];
    for (int a = 0; a < 3; a++)
        for (int ap = 0; ap < 3; ap++) {
            int idx = 3 * a + ap;
            int e = ((-2 * a * ap) % 3 + 3) % 3;
            /* w^e computed as a power of w, like the reference's w^exponent */
            cplx ph = {1, 0};
            for (int i = 0; i < e; i++) ph = cmul(ph, w);
            cplx ZX[9];
            mat3_mul(Zp[a], Xp[ap], ZX);
            for (int i = 0; i < 9; i++) T[idx][i] = cmul(ph, ZX[i]);
        }
    cplx A0[9] = {{0}};
    for (int u = 0; u < 9; u++)
        for (int i = 0; i < 9; i++) A0[i] = cadd(A0[i], T[u][i]);
    for (int i = 0; i < 9; i++) { A0[i].re /= 3.0; A0[i].im /= 3.0; }
    for (int idx = 0; idx < 9; idx++) {
        cplx Td[9], tmp[9], Au[9];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) Td[3 * i + j] = cconj(T[idx][3 * j + i]);
        mat3_mul(T[idx], A0, tmp);
        mat3_mul(tmp, Td, Au);
        /* vec(transpose(Au)) column-major: c = i + 3 j holds Au^T[i, j] = Au[j, i] */
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                int c = i + 3 * j;
                Mout[2 * (9 * idx + c)] = Au[3 * j + i].re;
                Mout[2 * (9 * idx + c) + 1] = Au[3 * j + i].im;
            }
    }
}

/* src/Mana.jl:190-228 (vec_rho_tensor_N) + 236-281 (apply_M_tensor_N_inplace!) +
 * 305-314 (Mana(rho)): v[p] = rho[r0, c0] with p's base-9 digit for site k (site 1 most
 * significant) = 3 i_k + j_k, i_k / j_k the k-th most significant ternary digits of r0 /
 * c0; w = M^{(x)N} v leg by leg (leg 1 = most significant digit); mana = log2(sum|w| /
 * 3^N).  rho is column-major interleaved complex: rho[r0 + dim*c0]. */
int or_mana_mixed(const double *rho, int N, double *mana_out, double *w_out) {
    if (N < 0 || N > 8) return OR_ERR_ARG;
    int64_t dim = 1, op = 1;
    for (int i = 0; i < N; i++) { dim *= 3; op *= 9; }
    double Mre[162];
    or_single_qutrit_M(Mre);
    cplx M[81];
    for (int i = 0; i < 81; i++) { M[i].re = Mre[2 * i]; M[i].im = Mre[2 * i + 1]; }
    cplx *v = calloc((size_t)op, sizeof(cplx));
    int idig[16], jdig[16];
    for (int64_t c0 = 0; c0 < dim; c0++) {
        int64_t t = c0;
        for (int k = N - 1; k >= 0; k--) { jdig[k] = (int)(t % 3); t /= 3; }
        for (int64_t r0 = 0; r0 < dim; r0++) {
            int64_t u = r0;
            for (int k = N - 1; k >= 0; k--) { idig[k] = (int)(u % 3); u /= 3; }
            int64_t p = 0;
            for (int k = 0; k < N; k++) p = p * 9 + (3 * idig[k] + jdig[k]);
            v[p].re = rho[2 * (r0 + dim * c0)];
            v[p].im = rho[2 * (r0 + dim * c0) + 1];
        }
    }
    cplx x[9], y[9];
    for (int leg = 1; leg <= N; leg++) {
        int64_t stride = 1;
        for (int i = 0; i < N - leg; i++) stride *= 9;
        int64_t block = stride * 9, nblocks = op / block;
        for (int64_t b = 0; b < nblocks; b++)
            for (int64_t ofs = 0; ofs < stride; ofs++) {
                int64_t base = b * block + ofs;
                for (int a = 0; a < 9; a++) x[a] = v[base + a * stride];
                for (int r = 0; r < 9; r++) {
                    cplx s = {0, 0};
                    for (int c = 0; c < 9; c++) s = cadd(s, cmul(M[9 * r + c], x[c]));
                    y[r] = s;
                }
                for (int a = 0; a < 9; a++) v[base + a * stride] = y[a];
            }
    }
    double s = 0.0;
    for (int64_t i = 0; i < op; i++) s += hypot(v[i].re, v[i].im);
    if (w_out)
        for (int64_t i = 0; i < op; i++) { w_out[2 * i] = v[i].re; w_out[2 * i + 1] = v[i].im; }
    *mana_out = log2(s / (double)dim);
    free(v);
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* Adjoint (no reference counterpart): d SRE / d(Re psi, Im psi)              */
/* ------------------------------------------------------------------------- */

/* Differentiates the reference's forward definition (src/SRE.jl:509-540 build,
 * FWHT, sum of (F^2)^q) directly: for each x, G_x = WHT(2q F^{2q-1}) and, with
 * s = r ^ x, g_x(r) = X1[r] T1[s] + X2[r] T2[s] (T1 = X1 + X2, T2 = X2 - X1):
 *   dm/dX1[r] += G(r) T1[s],  dm/dX2[r] += G(r) T2[s],
 *   dm/dX1[s] += G(r) (X1[r] - X2[r]),  dm/dX2[s] += G(r) (X1[r] + X2[r]).
 * dSRE = -dm / (m ln 2).  grad is interleaved (d/dRe, d/dIm).  The sums across X-strings
 * (m and every gradient entry) are double-double, so the only roundings left are those of
 * each X-string's own transform. */
int or_sre_grad(const double *psi, int n, double q, int nthreads, double *sre_out, double *grad) {
    if (n < 1 || n > 22 || nthreads < 1) return OR_ERR_ARG;
    sre_prep s;
    if (sre_prep_init(&s, psi, n) != OR_OK) return OR_ERR_ARG;
    const int64_t dim = s.dim;
    /* per thread: gradient (hi, lo) pairs, 4 doubles per amplitude */
    double *gacc = calloc((size_t)nthreads * 4 * (size_t)dim, sizeof(double));
    double *macc = calloc(2 * (size_t)nthreads, sizeof(double));
#pragma omp parallel num_threads(nthreads)
    {
        int tid = omp_get_thread_num();
        double *v = or_valloc(dim);
        double *G = or_valloc(dim);
        double *g = gacc + (size_t)tid * 4 * (size_t)dim;
        double mhi = 0.0, mlo = 0.0;
#pragma omp for schedule(static)
        for (int64_t x = 0; x < dim; x++) {
            for (int64_t r = 0; r < dim; r++) {
                uint64_t j = (uint64_t)r ^ (uint64_t)x;
                v[r] = fma(s.X1[r], s.TMP1[j], s.X2[r] * s.TMP2[j]);
            }
            or_fwht(v, n);
            double mx = 0.0;
            for (int64_t k = 0; k < dim; k++) {
                double F = v[k], p = F * F;
                mx += pow_q(p, q);
                /* d/dF (F^2)^q = 2 q F^(2q-1) = 2 q p^(q-1) F */
                G[k] = 2.0 * q * (q == 2.0 ? p : pow(p, q - 1.0)) * F;
            }
            dd_acc(&mhi, &mlo, mx);
            or_fwht(G, n);
            for (int64_t r = 0; r < dim; r++) {
                uint64_t sidx = (uint64_t)r ^ (uint64_t)x;
                double gr = G[r];
                dd_acc(&g[4 * r], &g[4 * r + 1], gr * s.TMP1[sidx]);
                dd_acc(&g[4 * r + 2], &g[4 * r + 3], gr * s.TMP2[sidx]);
                dd_acc(&g[4 * sidx], &g[4 * sidx + 1], gr * (s.X1[r] - s.X2[r]));
                dd_acc(&g[4 * sidx + 2], &g[4 * sidx + 3], gr * (s.X1[r] + s.X2[r]));
            }
        }
        macc[2 * tid] = mhi;
        macc[2 * tid + 1] = mlo;
        free(v);
        free(G);
    }
    double mh = 0.0, ml = 0.0;
    for (int t = 0; t < nthreads; t++) {
        dd_acc(&mh, &ml, macc[2 * t]);
        ml += macc[2 * t + 1];
    }
    const double m = mh + ml;
    const double scale = -1.0 / (m * log(2.0));
    for (int64_t i = 0; i < 2 * dim; i++) {
        double ah = 0.0, al = 0.0;
        for (int t = 0; t < nthreads; t++) {
            dd_acc(&ah, &al, gacc[(size_t)t * 4 * (size_t)dim + 2 * (size_t)i]);
            al += gacc[(size_t)t * 4 * (size_t)dim + 2 * (size_t)i + 1];
        }
        grad[i] = scale * (ah + al);
    }
    *sre_out = -log2(m / (double)dim);
    free(gacc);
    free(macc);
    sre_prep_free(&s);
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* State preparation (the step before the path)                                */
/* ------------------------------------------------------------------------- */

/* apply_2gate! of src/State.jl:254-345 (apply_2gate_qubit! 279-309, apply_2gate_qudit!
 * 311-344): for every input index i with digits d1 (site s1) and d2 (site s2), sites
 * 1-based with site 1 the least significant digit, idx_in = d1 q + d2, and for every
 * output o = o1 q + o2: tmp[base + o1 q^(s1-1) + o2 q^(s2-1)] += gate[o, idx_in] psi[i].
 * gate: q^2 x q^2 complex, column-major, interleaved (re, im).  psi: q^n complex,
 * interleaved, updated in place.  q in {2, 3}; s1 != s2 in [1, n]. */
int or_apply_2gate(double *psi, int n, int q, const double *gate, int s1, int s2) {
    if ((q != 2 && q != 3) || n < 2 || s1 < 1 || s2 < 1 || s1 > n || s2 > n || s1 == s2) return OR_ERR_ARG;
    int64_t N = 1;
    for (int k = 0; k < n; k++) N *= q;
    int64_t p1 = 1, p2 = 1;
    for (int k = 1; k < s1; k++) p1 *= q;
    for (int k = 1; k < s2; k++) p2 *= q;
    const int q2 = q * q;
    double *tmp = calloc((size_t)N * 2, sizeof(double));
    if (!tmp) return OR_ERR_ARG;
    for (int64_t i = 0; i < N; i++) {
        const double ar = psi[2 * i], ai = psi[2 * i + 1];
        const int64_t d1 = (i / p1) % q, d2 = (i / p2) % q;
        const int64_t idx_in = d1 * q + d2;
        const int64_t base = i - d1 * p1 - d2 * p2;
        for (int o = 0; o < q2; o++) {
            const int64_t j = base + (o / q) * p1 + (o % q) * p2;
            const double gr = gate[2 * (o + q2 * idx_in)], gi = gate[2 * (o + q2 * idx_in) + 1];
            tmp[2 * j] += gr * ar - gi * ai;
            tmp[2 * j + 1] += gr * ai + gi * ar;
        }
    }
    memcpy(psi, tmp, (size_t)N * 2 * sizeof(double));
    free(tmp);
    return OR_OK;
}

/* apply_brick_wall_haar! of src/State.jl:200-221 (and the layer pattern of
 * apply_brick_wall_cliff!, 146-183) with the gates given: layer l = 1..depth acts on
 * sites (s, s+1) for s = 1, 3, 5, ... (odd l) or s = 2, 4, ... (even l), s <= n - 1,
 * taking the next q^2 x q^2 gate of `gates` for every pair. */
int or_brick_wall(double *psi, int n, int q, int depth, const double *gates, int ngates) {
    const int q4 = q * q * q * q;
    int k = 0;
    for (int layer = 1; layer <= depth; layer++) {
        for (int s = (layer & 1) ? 1 : 2; s <= n - 1; s += 2) {
            if (k >= ngates) return OR_ERR_ARG;
            int rc = or_apply_2gate(psi, n, q, gates + (size_t)2 * q4 * k, s, s + 1);
            if (rc != OR_OK) return rc;
            k++;
        }
    }
    return k == ngates ? OR_OK : OR_ERR_ARG;
}

/* reduced_density_matrix of src/DensityMatrix.jl:94-123 (rho_A = Tr_B |psi><psi|):
 * side 0 (:left) keeps sites 1..NA,  rho[iA, jA] = sum_kB psi[iA + dimA kB] conj(psi[jA + dimA kB]);
 * side 1 (:right) keeps sites N-NA+1..N, rho[iA, jA] = sum_kB psi[iA dimB + kB] conj(psi[jA dimB + kB]).
 * rho: dimA x dimA complex, column-major, interleaved. */
int or_reduced_density_matrix(const double *psi, int n, int q, int NA, int side, double *rho) {
    if ((q != 2 && q != 3) || NA < 0 || NA > n || (side != 0 && side != 1)) return OR_ERR_ARG;
    int64_t dimA = 1, dimB = 1;
    for (int k = 0; k < NA; k++) dimA *= q;
    for (int k = 0; k < n - NA; k++) dimB *= q;
#pragma omp parallel for schedule(static)
    for (int64_t jA = 0; jA < dimA; jA++) {
        for (int64_t iA = 0; iA < dimA; iA++) {
            double sr = 0.0, si = 0.0;
            for (int64_t kB = 0; kB < dimB; kB++) {
                const int64_t a = side == 0 ? iA + dimA * kB : iA * dimB + kB;
                const int64_t b = side == 0 ? jA + dimA * kB : jA * dimB + kB;
                const double ar = psi[2 * a], ai = psi[2 * a + 1], br = psi[2 * b], bi = psi[2 * b + 1];
                sr += ar * br + ai * bi;
                si += ai * br - ar * bi;
            }
            rho[2 * (iA + dimA * jA)] = sr;
            rho[2 * (iA + dimA * jA) + 1] = si;
        }
    }
    return OR_OK;
}
