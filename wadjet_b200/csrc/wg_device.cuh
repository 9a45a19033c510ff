// wg_device.cuh — device helpers shared by the kernels of libwadjetgpu.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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

#define WG_FULL_MASK 0xFFFFFFFFu

namespace wgd {

struct DCol {
  const void* data;
  const uint64_t* valid;   // nullptr = no nulls
  int32_t cls;
  int32_t scale;
};

__device__ __forceinline__ bool is_null(const DCol& c, int64_t i) {
  return c.valid != nullptr && ((__ldg(&c.valid[i >> 6]) >> (i & 63)) & 1ULL) == 0;
}

__device__ __forceinline__ int64_t ld_i64(const DCol& c, int64_t i) {
  return c.cls == WG_CLS_I32 ? (int64_t)__ldg((const int32_t*)c.data + i) : __ldg((const long long*)c.data + i);
}

// math.Pow10 as Go computes it for n in [0, 128): pow10tab[n%32] * pow10postab32[n/32]
static __constant__ double c_pow10_tab[32] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10,
                                              1e11, 1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21,
                                              1e22, 1e23, 1e24, 1e25, 1e26, 1e27, 1e28, 1e29, 1e30, 1e31};
static __constant__ double c_pow10_post[4] = {1e0, 1e32, 1e64, 1e96};
__device__ __forceinline__ double pow10_go(int n) {
  if (n < 0 || n >= 128) return 1.0;
  return __dmul_rn(c_pow10_tab[n & 31], c_pow10_post[n >> 5]);
}

// Int128.ToFloat64 (internal/engine/batch/decimal.go:39-51), IEEE round-to-nearest
// at every step and no contraction, so the result is Go's bit for bit.
__device__ __forceinline__ double dec_to_f64(int64_t hi, uint64_t lo, int scale) {
  if ((hi == 0 && lo <= 0x7FFFFFFFFFFFFFFFULL) || (hi == -1 && lo > 0x7FFFFFFFFFFFFFFFULL))
    return __ddiv_rn(__ll2double_rn((long long)lo), pow10_go(scale));
  double f = __dadd_rn(__dmul_rn(__ll2double_rn(hi), 18446744073709551616.0), __ull2double_rn(lo));
  return __ddiv_rn(f, pow10_go(scale));
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

__device__ __forceinline__ void atomic_min128(U128* p, unsigned long long lo, unsigned long long hi) {
  U128 cur = read128(p);
  while (less128(lo, hi, cur.lo, cur.hi)) {
    U128 nv; nv.lo = lo; nv.hi = hi;
    U128 old = cas128(p, cur, nv);
    if (old.lo == cur.lo && old.hi == cur.hi) return;
    cur = old;
  }
}
__device__ __forceinline__ void atomic_max128(U128* p, unsigned long long lo, unsigned long long hi) {
  U128 cur = read128(p);
  while (less128(cur.lo, cur.hi, lo, hi)) {
    U128 nv; nv.lo = lo; nv.hi = hi;
    U128 old = cas128(p, cur, nv);
    if (old.lo == cur.lo && old.hi == cur.hi) return;
    cur = old;
  }
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
