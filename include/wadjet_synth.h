/*
 * wadjet_synth.h — seeded, counter-based synthetic tables for the benchmark
 * workloads (no public dataset is used; these generators stand in for them).
 *
 * Every value is a pure function of (seed, stream, row), so a row can be
 * produced independently on the GPU (one thread per row) or on the CPU, and the
 * two agree bit for bit: only integer arithmetic, exact binary64 scaling by
 * powers of two, single IEEE additions/multiplications, and comparisons against
 * a host-built table. No transcendental function is evaluated per row.
 *
 * Workloads (sizes are parameters; defaults are the benchmark shapes):
 *  - groupby:  k int64 U[0,4096), v int64 U[0,1e6), f float64 U[0,1),
 *              flag int32 U[0,10)   — SELECT k,SUM(v),COUNT(*),MIN(f),MAX(f)
 *              WHERE flag < 7 GROUP BY k.
 *  - starjoin: fact fk int32 Zipf(s=1.1) over 2^22 keys, qty int32 U[1,50],
 *              price DECIMAL(15,2) U[1.00, 100000.00] as Int128 cents,
 *              disc float64 U[0,0.1); dimension of 2^22 unique int32 keys
 *              (a fixed permutation of 0..2^22-1) with grp int32 U[0,1000).
 *  - highcard: b int64 = bijective scramble of U[0,2^26), a int32 = 16 bits of
 *              a second scramble of b (so (a,b) takes ~2^26 values), amount
 *              DECIMAL(18,2) U[-1e6, 1e6] as Int128 cents, x float64 ≈ N(0,1)
 *              as an Irwin–Hall sum of 12 uniforms minus 6.
 *
 * Generator: SplitMix64 (Steele, Lea & Flood, "Fast splittable pseudorandom
 * number generators", OOPSLA 2014) — state = stream_seed + row * golden gamma,
 * output = the SplitMix64 finalizer of the state. Bounded integers use the
 * multiply-high mapping (Lemire 2019) without rejection.
 */
#ifndef WADJET_SYNTH_H
#define WADJET_SYNTH_H

#include <stdint.h>

#if defined(__CUDACC__)
#define WG_SYN_HD __host__ __device__ __forceinline__
#else
#define WG_SYN_HD static inline
#endif

#define WG_SYN_DEFAULT_SEED 42ULL

/* streams (one per generated column) */
#define WG_SYN_GB_K      1
#define WG_SYN_GB_V      2
#define WG_SYN_GB_F      3
#define WG_SYN_GB_FLAG   4
#define WG_SYN_SJ_FK    10
#define WG_SYN_SJ_QTY   11
#define WG_SYN_SJ_PRICE 12
#define WG_SYN_SJ_DISC  13
#define WG_SYN_SJ_GRP   14
#define WG_SYN_HC_B     20
#define WG_SYN_HC_AMT   21
#define WG_SYN_HC_X0    22   /* 22..33: the 12 uniforms of x */

#define WG_SYN_SJ_DIM_BITS 22                       /* 4,194,304 keys */
#define WG_SYN_SJ_ZIPF_S   1.1
#define WG_SYN_HC_B_BITS   26

WG_SYN_HD uint64_t wg_syn_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

WG_SYN_HD uint64_t wg_syn_u64(uint64_t seed, uint32_t stream, uint64_t row) {
  uint64_t base = wg_syn_mix64(seed ^ ((uint64_t)stream * 0xD1B54A32D192ED03ULL));
  return wg_syn_mix64(base + row * 0x9E3779B97F4A7C15ULL);
}

WG_SYN_HD uint64_t wg_syn_mulhi(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
#endif
}

/* uniform integer in [lo, hi] (inclusive) */
WG_SYN_HD int64_t wg_syn_int(uint64_t seed, uint32_t stream, uint64_t row, int64_t lo, int64_t hi) {
  uint64_t range = (uint64_t)(hi - lo) + 1ULL;
  return lo + (int64_t)wg_syn_mulhi(wg_syn_u64(seed, stream, row), range);
}

/* uniform binary64 in [0, 1): 53 random bits times 2^-53 (exact) */
WG_SYN_HD double wg_syn_u01(uint64_t seed, uint32_t stream, uint64_t row) {
  return (double)(wg_syn_u64(seed, stream, row) >> 11) * (1.0 / 9007199254740992.0);
}

/* bijections of [0, 2^bits): odd multiplier plus offset modulo 2^bits */
WG_SYN_HD uint32_t wg_syn_perm_fact(uint32_t r, int bits) {
  return (uint32_t)((r * 0x9E3779B1u + 0x5BD1E995u) & ((1u << bits) - 1u));
}
WG_SYN_HD uint32_t wg_syn_perm_dim(uint32_t i, int bits) {
  return (uint32_t)((i * 0x2545F491u + 0x3C6EF372u) & ((1u << bits) - 1u));
}

/* smallest index i with cdf[i] > u (cdf ascending, cdf[n-1] == 1.0) */
WG_SYN_HD int64_t wg_syn_cdf_search(const double* cdf, int64_t n, double u) {
  int64_t lo = 0, hi = n - 1;
  while (lo < hi) {
    int64_t mid = lo + ((hi - lo) >> 1);
    if (cdf[mid] > u) hi = mid; else lo = mid + 1;
  }
  return lo;
}

/* ---- starjoin columns ---- */
WG_SYN_HD int32_t wg_syn_sj_fk(uint64_t seed, uint64_t row, const double* cdf, int bits) {
  double u = wg_syn_u01(seed, WG_SYN_SJ_FK, row);
  int64_t rank = wg_syn_cdf_search(cdf, (int64_t)1 << bits, u);
  return (int32_t)wg_syn_perm_fact((uint32_t)rank, bits);
}
WG_SYN_HD int32_t wg_syn_sj_qty(uint64_t seed, uint64_t row) {
  return (int32_t)wg_syn_int(seed, WG_SYN_SJ_QTY, row, 1, 50);
}
/* price cents in [100, 10,000,000]: DECIMAL(15,2) 1.00 .. 100000.00 */
WG_SYN_HD int64_t wg_syn_sj_price(uint64_t seed, uint64_t row) {
  return wg_syn_int(seed, WG_SYN_SJ_PRICE, row, 100, 10000000);
}
WG_SYN_HD double wg_syn_sj_disc(uint64_t seed, uint64_t row) {
  return wg_syn_u01(seed, WG_SYN_SJ_DISC, row) * 0.1;
}
WG_SYN_HD int32_t wg_syn_sj_dim_key(uint64_t i, int bits) {
  return (int32_t)wg_syn_perm_dim((uint32_t)i, bits);
}
WG_SYN_HD int32_t wg_syn_sj_grp(uint64_t seed, uint64_t i) {
  return (int32_t)wg_syn_int(seed, WG_SYN_SJ_GRP, i, 0, 999);
}

/* ---- groupby columns ---- */
WG_SYN_HD int64_t wg_syn_gb_k(uint64_t seed, uint64_t row, int64_t ngroups) {
  return wg_syn_int(seed, WG_SYN_GB_K, row, 0, ngroups - 1);
}
WG_SYN_HD int64_t wg_syn_gb_v(uint64_t seed, uint64_t row) {
  return wg_syn_int(seed, WG_SYN_GB_V, row, 0, 999999);
}
WG_SYN_HD double wg_syn_gb_f(uint64_t seed, uint64_t row) {
  return wg_syn_u01(seed, WG_SYN_GB_F, row);
}
WG_SYN_HD int32_t wg_syn_gb_flag(uint64_t seed, uint64_t row) {
  return (int32_t)wg_syn_int(seed, WG_SYN_GB_FLAG, row, 0, 9);
}

/* ---- highcard columns ---- */
WG_SYN_HD int64_t wg_syn_hc_b(uint64_t seed, uint64_t row, int bits) {
  uint64_t v = (uint64_t)wg_syn_int(seed, WG_SYN_HC_B, row, 0, ((int64_t)1 << bits) - 1);
  return (int64_t)wg_syn_mix64(v ^ 0x6A09E667F3BCC909ULL);
}
WG_SYN_HD int32_t wg_syn_hc_a(int64_t b) {
  return (int32_t)(wg_syn_mix64((uint64_t)b ^ 0xBB67AE8584CAA73BULL) & 0xFFFFULL);
}
/* amount cents in [-1e8, 1e8]: DECIMAL(18,2) -1e6 .. 1e6 */
WG_SYN_HD int64_t wg_syn_hc_amt(uint64_t seed, uint64_t row) {
  return wg_syn_int(seed, WG_SYN_HC_AMT, row, -100000000LL, 100000000LL);
}
WG_SYN_HD double wg_syn_hc_x(uint64_t seed, uint64_t row) {
  double s = 0.0;
  for (uint32_t j = 0; j < 12; ++j) s = s + wg_syn_u01(seed, WG_SYN_HC_X0 + j, row);
  return s - 6.0;
}

/* ---- batched workload: query q of a batch ----
 * rows N_q = round(exp(U[ln 1e4, ln 1e7])), key cardinality C_q =
 * round(exp(U[ln 16, ln 1e6])), selectivity s_q ~ U[0.1, 0.9] → filter
 * `f < round(1000 s_q)` on f int32 U[0,1000); value int64 U[0,1e6) for even q,
 * float64 U[0,1) for odd q; key int64 U[0, C_q). Rows use seed + q. */
#define WG_SYN_BQ_KEY   40
#define WG_SYN_BQ_VI    41
#define WG_SYN_BQ_VF    42
#define WG_SYN_BQ_FILT  43
#define WG_SYN_BQ_PARAM 44

WG_SYN_HD int64_t wg_syn_bq_key(uint64_t seed, uint64_t row, int64_t card) {
  return wg_syn_int(seed, WG_SYN_BQ_KEY, row, 0, card - 1);
}
WG_SYN_HD int64_t wg_syn_bq_vi(uint64_t seed, uint64_t row) { return wg_syn_int(seed, WG_SYN_BQ_VI, row, 0, 999999); }
WG_SYN_HD double wg_syn_bq_vf(uint64_t seed, uint64_t row) { return wg_syn_u01(seed, WG_SYN_BQ_VF, row); }
WG_SYN_HD int32_t wg_syn_bq_filt(uint64_t seed, uint64_t row) {
  return (int32_t)wg_syn_int(seed, WG_SYN_BQ_FILT, row, 0, 999);
}

#include <math.h>
#if defined(__CUDACC__)
#define WG_SYN_HOST __host__ static inline
#else
#define WG_SYN_HOST static inline
#endif

/* Parameters of query q (host only: uses exp/log once per query). */
WG_SYN_HOST void wg_syn_bq_params(uint64_t seed, uint32_t q, int64_t* rows, int64_t* card, int32_t* threshold) {
  const double u0 = wg_syn_u01(seed, WG_SYN_BQ_PARAM, 3ULL * q);
  const double u1 = wg_syn_u01(seed, WG_SYN_BQ_PARAM, 3ULL * q + 1);
  const double u2 = wg_syn_u01(seed, WG_SYN_BQ_PARAM, 3ULL * q + 2);
  *rows = (int64_t)llround(exp(log(1e4) + u0 * (log(1e7) - log(1e4))));
  *card = (int64_t)llround(exp(log(16.0) + u1 * (log(1e6) - log(16.0))));
  *threshold = (int32_t)llround(1000.0 * (0.1 + 0.8 * u2));
}
/* Zipf(s) inverse-CDF table over n ranks: cdf[i] = sum_{r<=i} (r+1)^-s / total,
 * summed in rank order, last entry forced to exactly 1.0. Built once on the
 * host and shared by every consumer so all of them sample identical keys. */
WG_SYN_HOST void wg_syn_zipf_cdf(double* cdf, int64_t n, double s) {
  double acc = 0.0;
  for (int64_t r = 0; r < n; ++r) {
    acc += pow((double)(r + 1), -s);
    cdf[r] = acc;
  }
  for (int64_t r = 0; r < n; ++r) cdf[r] = cdf[r] / acc;
  cdf[n - 1] = 1.0;
}

#endif /* WADJET_SYNTH_H */
