// wg_device.cuh — device helpers shared by the kernels of libwadjetgpu.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "wadjet_gpu.h"

// storage classes of the column types the GPU path reads
#define WG_CLS_I32 0   // Int32Data: INT32, PORT, PROTOCOL, DATE
#define WG_CLS_I64 1   // Int64Data: INT64, TIMESTAMP, IPV4, MAC, DURATION
#define WG_CLS_F32 2
#define WG_CLS_F64 3
#define WG_CLS_DEC 4   // DecimalData: {int64 hi; uint64 lo}
#define WG_CLS_BAD 5

// device-side error codes written to the context's error word
#define WG_DERR_NONE        0
#define WG_DERR_TABLE_FULL  1   // a hash probe walked the whole table
#define WG_DERR_TIMEOUT     2   // a bounded wait gave up
#define WG_DERR_NULL_PACKED 3   // NULL in a composite (packed) group key
#define WG_DERR_STACK       4   // malformed expression program
#define WG_DERR_BAD_PAGE    5   // a Parquet page whose levels, indices or values are malformed
#define WG_DERR_HASH_COLLISION 6  // two different strings with one 128-bit dictionary hash

#define WG_FULL_MASK 0xFFFFFFFFu

namespace wgd {

struct DCol {
  const void* data;
  const uint64_t* valid;   // nullptr = no nulls
  int32_t cls;
  int32_t scale;
};

// Read-only loads that ask L2 to keep their lines (evict-last) while streamed
// data passes through: for small tables probed once per streamed row.
__device__ __forceinline__ uint64_t l2_keep_policy() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint32_t ld_keep_u32(const uint32_t* p) {
  uint32_t v;
  asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(l2_keep_policy()));
  return v;
}
__device__ __forceinline__ unsigned long long ld_keep_u64(const unsigned long long* p) {
  unsigned long long v;
  asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(l2_keep_policy()));
  return v;
}

__device__ __forceinline__ bool is_null(const DCol& c, int64_t i) {
  return c.valid != nullptr && ((__ldg(&c.valid[i >> 6]) >> (i & 63)) & 1ULL) == 0;
}

__device__ __forceinline__ int64_t ld_i64(const DCol& c, int64_t i) {
  return c.cls == WG_CLS_I32 ? (int64_t)__ldg((const int32_t*)c.data + i) : __ldg((const long long*)c.data + i);
}

// math.Pow10 as Go computes it for n in [0, 128): pow10tab[n%32] * pow10postab32[n/32]
#define WG_POW10_TAB 1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11, 1e12, 1e13, 1e14, \
                     1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22, 1e23, 1e24, 1e25, 1e26, 1e27, 1e28, 1e29, 1e30, 1e31
#define WG_POW10_POST 1e0, 1e32, 1e64, 1e96
static __constant__ double c_pow10_tab[32] = {WG_POW10_TAB};
static __constant__ double c_pow10_post[4] = {WG_POW10_POST};
__device__ __forceinline__ double pow10_go(int n) {
  if (n < 0 || n >= 128) return 1.0;
  return __dmul_rn(c_pow10_tab[n & 31], c_pow10_post[n >> 5]);
}

// RN(1 / pow10_go(n)) for n in [0, 128), as exact binary64 literals.
#define WG_POW10_RECIP \
    0x1.0000000000000p+0, 0x1.999999999999ap-4, 0x1.47ae147ae147bp-7, 0x1.0624dd2f1a9fcp-10, \
    0x1.a36e2eb1c432dp-14, 0x1.4f8b588e368f1p-17, 0x1.0c6f7a0b5ed8dp-20, 0x1.ad7f29abcaf48p-24, \
    0x1.5798ee2308c3ap-27, 0x1.12e0be826d695p-30, 0x1.b7cdfd9d7bdbbp-34, 0x1.5fd7fe1796495p-37, \
    0x1.19799812dea11p-40, 0x1.c25c268497682p-44, 0x1.6849b86a12b9bp-47, 0x1.203af9ee75616p-50, \
    0x1.cd2b297d889bcp-54, 0x1.70ef54646d497p-57, 0x1.2725dd1d243acp-60, 0x1.d83c94fb6d2acp-64, \
    0x1.79ca10c924223p-67, 0x1.2e3b40a0e9b4fp-70, 0x1.e392010175ee6p-74, 0x1.82db34012b252p-77, \
    0x1.357c299a88ea8p-80, 0x1.ef2d0f5da7dd8p-84, 0x1.8c240c4aecb13p-87, 0x1.3ce9a36f23c10p-90, \
    0x1.fb0f6be50601ap-94, 0x1.95a5efea6b348p-97, 0x1.4484bfeebc29fp-100, 0x1.039d665896880p-103, \
    0x1.9f623d5a8a732p-107, 0x1.4c4e977ba1f5bp-110, 0x1.09d8792fb4c49p-113, 0x1.a95a5b7f87a0fp-117, \
    0x1.54484932d2e72p-120, 0x1.1039d428a8b8ep-123, 0x1.b38fb9daa78e4p-127, 0x1.5c72fb1552d83p-130, \
    0x1.16c262777579cp-133, 0x1.be03d0bf225c7p-137, 0x1.64cfda3281e38p-140, 0x1.1d7314f534b61p-143, \
    0x1.c8b8218854567p-147, 0x1.6d601ad376ab9p-150, 0x1.244ce242c5561p-153, 0x1.d3ae36d13bbcep-157, \
    0x1.7624f8a762fd8p-160, 0x1.2b50c6ec4f313p-163, 0x1.dee7a4ad4b81ep-167, 0x1.7f1fb6f10934cp-170, \
    0x1.327fc58da0f70p-173, 0x1.ea6608e29b24dp-177, 0x1.8851a0b548ea3p-180, 0x1.39dae6f76d883p-183, \
    0x1.f62b0b257c0d1p-187, 0x1.91bc08eac9a40p-190, 0x1.41633a556e1cdp-193, 0x1.011c2eaabe7d8p-196, \
    0x1.9b604aaaca627p-200, 0x1.4919d5556eb52p-203, 0x1.0747ddddf22a8p-206, 0x1.a53fc9631d10cp-210, \
    0x1.50ffd44f4a73dp-213, 0x1.0d9976a5d5297p-216, 0x1.af5bf109550f3p-220, 0x1.59165a6ddda5bp-223, \
    0x1.1411e1f17e1e2p-226, 0x1.b9b6364f30304p-230, 0x1.615e91d8f359dp-233, 0x1.1ab20e472914ap-236, \
    0x1.c45016d841babp-240, 0x1.69d9abe034955p-243, 0x1.217aefe690777p-246, 0x1.cf2b1970e7259p-250, \
    0x1.7288e1271f513p-253, 0x1.286d80ec190dcp-256, 0x1.da48ce468e7c7p-260, 0x1.7b6d71d20b96cp-263, \
    0x1.2f8ac174d6123p-266, 0x1.e5aacf2156839p-270, 0x1.8488a5b445361p-273, 0x1.36d3b7c36a91ap-276, \
    0x1.f152bf9f10e8fp-280, 0x1.8ddbcc7f40ba6p-283, 0x1.3e497065cd61ep-286, 0x1.fd424d6faf031p-290, \
    0x1.97683df2f268ep-293, 0x1.45ecfe5bf520ap-296, 0x1.04bd984990e6fp-299, 0x1.a12f5a0f4e3e4p-303, \
    0x1.4dbf7b3f71cb7p-306, 0x1.0aff95cc5b093p-309, 0x1.ab328946f80eap-313, 0x1.55c2076bf9a55p-316, \
    0x1.116805effaeaap-319, 0x1.b5733cb32b110p-323, 0x1.5df5ca28ef40dp-326, 0x1.17f7d4ed8c33dp-329, \
    0x1.bff2ee48e0530p-333, 0x1.665bf1d3e6a8dp-336, 0x1.1eaff4a98553dp-339, 0x1.cab3210f3bb95p-343, \
    0x1.6ef5b40c2fc77p-346, 0x1.25915cd68c9f9p-349, 0x1.d5b561574765bp-353, 0x1.77c44ddf6c516p-356, \
    0x1.2c9d0b1923745p-359, 0x1.e0fb44f50586ep-363, 0x1.80c903f7379f1p-366, 0x1.33d4032c2c7f4p-369, \
    0x1.ec866b79e0cb9p-373, 0x1.8a0522c7e7095p-376, 0x1.3b374f06526dep-379, 0x1.f8587e7083e2fp-383, \
    0x1.9379fec069826p-386, 0x1.42c7ff0054685p-389, 0x1.023998cd10537p-392, 0x1.9d28f47b4d525p-396, \
    0x1.4a8729fc3ddb7p-399, 0x1.086c219697e2bp-402, 0x1.a71368f0f3046p-406, 0x1.5275ed8d8f36bp-409, \
    0x1.0ec4be0ad8f89p-412, 0x1.b13ac9aaf4c0fp-416, 0x1.5a956e225d672p-419, 0x1.1544581b7dec2p-422
static __constant__ double c_pow10_recip[128] = {WG_POW10_RECIP};

// a / b correctly rounded given y = RN(1/b) (b = pow10_go(n) for div_pow10),
// without a division: Markstein's
// correction (P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990): with y = RN(1/b)
// and q within one ulp of a/b, the remainder r = a - b*q is exact in one FMA
// and RN(q + r*y) is RN(a/b). q = RN(a*y) can be up to 1.5 ulp off, so one
// correction brings it within one ulp and a second one makes it exact. Valid
// while nothing overflows or underflows: |a| < 2^128 and b <= 1e127 here.
__device__ __forceinline__ double div_by_recip(double a, double b, double y) {
  double q = __dmul_rn(a, y);
  double r = __fma_rn(-q, b, a);
  q = __fma_rn(r, y, q);
  r = __fma_rn(-q, b, a);
  return __fma_rn(r, y, q);
}

__device__ __forceinline__ double div_pow10(double a, int n) {
  if (n <= 0 || n >= 128) return a;  // pow10_go is 1 there
  return div_by_recip(a, pow10_go(n), c_pow10_recip[n]);
}

// The divisor pair div_pow10 uses for scale n, for a plan to carry per column:
// b = pow10_go(n), y = RN(1/b); b = y = 1 outside (0, 128), where the
// correction steps then return the dividend unchanged.
inline void pow10_divisor_host(int n, double* b, double* y) {
  static const double tab[32] = {WG_POW10_TAB}, post[4] = {WG_POW10_POST}, recip[128] = {WG_POW10_RECIP};
  if (n <= 0 || n >= 128) { *b = 1.0; *y = 1.0; return; }
  *b = tab[n & 31] * post[n >> 5];  // one IEEE product, as pow10_go
  *y = recip[n];
}

// Int128 to float64 before the scale division, as decimal.go:39-51 does
__device__ __forceinline__ double int128_to_f64(int64_t hi, uint64_t lo) {
  if (hi == ((long long)lo >> 63)) return __ll2double_rn((long long)lo);  // fits int64
  return __dadd_rn(__dmul_rn(__ll2double_rn(hi), 18446744073709551616.0), __ull2double_rn(lo));
}

// Int128.ToFloat64 (internal/engine/batch/decimal.go:39-51), IEEE round-to-nearest
// at every step and no contraction, so the result is Go's bit for bit.
__device__ __forceinline__ double dec_to_f64(int64_t hi, uint64_t lo, int scale) {
  return div_pow10(int128_to_f64(hi, lo), scale);
}

// expr.ColRef.EvalFloat64 (internal/engine/expr/expr.go:206-228)
__device__ __forceinline__ double ld_f64(const DCol& c, int64_t i) {
  switch (c.cls) {
    case WG_CLS_I32: return __ll2double_rn(__ldg((const int32_t*)c.data + i));
    case WG_CLS_I64: return __ll2double_rn(__ldg((const long long*)c.data + i));
    case WG_CLS_F32: return (double)__ldg((const float*)c.data + i);
    case WG_CLS_F64: return __ldg((const double*)c.data + i);
    case WG_CLS_DEC: {
      const longlong2 v = __ldg((const longlong2*)c.data + i);  // .x = hi, .y = lo
      return dec_to_f64(v.x, (uint64_t)v.y, c.scale);
    }
    default: return 0.0;
  }
}

// Order-preserving map of binary64 onto uint64 (negatives reversed below
// positives), so integer atomicMin/atomicMax give the float MIN/MAX.
__device__ __forceinline__ uint64_t f64_to_ord(double d) {
  uint64_t b = (uint64_t)__double_as_longlong(d);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __host__ __forceinline__ double ord_to_f64(uint64_t o) {
  uint64_t b = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFULL) : ~o;
  double d;
  memcpy(&d, &b, 8);
  return d;
}

// 128-bit two's-complement helpers on (lo, hi) words
__device__ __forceinline__ void add128(unsigned long long& lo, unsigned long long& hi, unsigned long long blo,
                                       unsigned long long bhi) {
  unsigned long long l = lo + blo;
  hi = hi + bhi + (l < lo ? 1ULL : 0ULL);
  lo = l;
}
__device__ __forceinline__ bool less128(unsigned long long alo, unsigned long long ahi, unsigned long long blo,
                                        unsigned long long bhi) {
  if (ahi != bhi) return (long long)ahi < (long long)bhi;
  return alo < blo;
}

// Exact Int128 accumulation with two 64-bit atomics: the low word's carry is
// read from the value it replaced, so the final (lo, hi) is the exact sum mod
// 2^128 whatever the interleaving. p[0] = lo, p[1] = hi.
__device__ __forceinline__ void atomic_add128(unsigned long long* p, unsigned long long lo, unsigned long long hi) {
  if (lo != 0) {
    unsigned long long old = atomicAdd(p, (unsigned long long)lo);
    if (old + lo < old) hi += 1;
  }
  if (hi != 0) atomicAdd(p + 1, (unsigned long long)hi);
}

struct __align__(16) U128 {
  unsigned long long lo, hi;
};

// 16-byte compare-and-swap (sm_90+ hardware 128-bit atomics)
__device__ __forceinline__ U128 cas128(U128* p, U128 cmp, U128 val) { return atomicCAS(p, cmp, val); }

// Two 64-bit volatile reads of a 16-byte slot. The pair may be torn (one word
// from before a concurrent CAS, one after); callers only act on it through a
// 128-bit CAS, which compares against the true value, or after checking that
// neither word can belong to the slot's previous state.
__device__ __forceinline__ U128 read128(const void* p) {
  const volatile unsigned long long* q = (const volatile unsigned long long*)p;
  U128 r;
  r.lo = q[0];
  r.hi = q[1];
  return r;
}

// Int128 MIN / MAX by 16-byte CAS. The first read may be torn, so a verdict of
// "no change needed" taken from it is confirmed by a CAS that writes the value
// it compares against (a no-op when the read was whole); every value returned
// by a CAS is the slot's true contents.
template <bool MIN>
__device__ __forceinline__ void atomic_minmax128(U128* p, unsigned long long lo, unsigned long long hi) {
  U128 cur = read128(p);
  bool whole = false;
  U128 nv; nv.lo = lo; nv.hi = hi;
  for (;;) {
    const bool better = MIN ? less128(lo, hi, cur.lo, cur.hi) : less128(cur.lo, cur.hi, lo, hi);
    if (!better && whole) return;
    const U128 old = cas128(p, cur, better ? nv : cur);
    if (old.lo == cur.lo && old.hi == cur.hi) return;
    cur = old;
    whole = true;
  }
}
__device__ __forceinline__ void atomic_min128(U128* p, unsigned long long lo, unsigned long long hi) {
  atomic_minmax128<true>(p, lo, hi);
}
__device__ __forceinline__ void atomic_max128(U128* p, unsigned long long lo, unsigned long long hi) {
  atomic_minmax128<false>(p, lo, hi);
}

// Fibonacci hashing on the high bits (Knuth 6.4): slot = (k * 2^64/phi) >> (64 - log2 cap)
__device__ __host__ __forceinline__ uint64_t fib_slot(uint64_t k, int shift) {
  return (k * 0x9E3779B97F4A7C15ULL) >> shift;
}
// 128-bit key fold (full-product halves xor'd, as packedHash in
// internal/engine/exec/packed_hash.go:155 does), then Fibonacci on the high bits
__device__ __forceinline__ uint64_t packed_slot(uint64_t lo, uint64_t hi, int shift) {
  uint64_t a = lo ^ 0x9E3779B97F4A7C15ULL, b = hi ^ 0x517CC1B727220A95ULL;
  uint64_t h = __umul64hi(a, b) ^ (a * b) ^ (lo + hi);
  return fib_slot(h, shift);
}

__device__ __forceinline__ void set_error(int32_t* err, int32_t code) {
  if (err) atomicCAS(err, 0, code);
}

}  // namespace wgd
