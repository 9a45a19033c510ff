// wg_join.cuh — device view of a built hash-join index, shared by the
// standalone probe and the fused filter → probe → aggregate kernel.
//
// The index restates HashJoin's int-key build (internal/engine/exec/join.go:
// 520-575): an open-addressing table maps each distinct key to the most
// recently inserted build row (the chain head) and `next[row]` links each build
// row to the previous row with the same key (arenaNext). Keys are widened to
// int64 as intKeyFromVector does (join.go:504). NULL keys are never indexed.
//
// Two slot flavours, picked from the build key's storage class:
//  - int32-class keys: one 8-byte word {key32 (low), head32 (high)}, so a
//    single 64-bit atomicCAS installs key and head together;
//  - int64-class keys: 16 bytes {key64, head32, pad32}, installed with the
//    sm_90+ 16-byte atomicCAS.
// A slot is empty when its head is -1 (every occupied slot has head >= 0).
#pragma once

#include "wadjet_gpu.h"
#include "wg_device.cuh"

#define WG_MAX_PAYLOAD 4

namespace wgd {

struct JoinView {
  int32_t flavor;          // 0 = 8-byte slots (int32 keys), 1 = 16-byte slots (int64 keys)
  int32_t shift;           // 64 - log2(capacity)
  uint64_t mask;           // capacity - 1
  const void* slots;
  const int32_t* next;
  int32_t n_pay;
  // Direct-payload table (unique int32 keys, one 4-byte payload without NULLs):
  // each slot holds {key32, payload32} instead of {key32, head32}, so a probe
  // returns the payload with one load; empty slots hold `sentinel`, an int32
  // that is not a build key.
  int32_t direct;
  int32_t sentinel;
  // Dense direct table (unique keys spanning a range at most a few times the
  // build size): slot i holds key base+i, so a probe is one load with no hash
  // and no probing; `mask` then holds the number of slots. dense = 2: every
  // key of the range is present, so `slots` is just the 4-byte payloads
  // (payload of key base+i at i) and a key in range always matches.
  int32_t dense;
  int32_t l2keep;          // dense probes ask L2 to keep the table's lines (evict-last)
  // exec.JoinType of the probe (join.go:20-30): WG_JOIN_INNER, WG_JOIN_LEFT
  // (an unmatched probe row once, with NULL build columns), WG_JOIN_SEMI (a
  // matched probe row once, no build columns), WG_JOIN_ANTI (a probe row with
  // no match or a NULL key, no build columns)
  int32_t jtype;
  // A pass over a partitioned build (one group of its key-hash partitions):
  // only probe rows whose key falls in partitions [part_lo, part_hi) take part
  // (partition = (key * fib) >> part_shift; NULL keys belong to the pass that
  // starts at partition 0). part_shift = 0: no partitioning.
  int32_t part_shift;
  int32_t part_lo, part_hi;
  long long base;
  DCol pay[WG_MAX_PAYLOAD];
  // Bloom pre-filter of the hash probe (nullptr: none): a key the bloom rules
  // out misses without reading the index (bloom_contains below).
  const unsigned long long* bloom;
  unsigned long long bloom_mask;
};

// HashJoin.buildBloom (join.go:1441) / BloomFilterOp (bloom_filter_op.go):
// bloomHashInt (join.go:1650), and the two bits bloomSet / bloomContains
// (bloom_filter_op.go:268) take from it in a table of 64-bit words.
__host__ __device__ __forceinline__ unsigned long long bloom_hash_int(long long key) {
  const unsigned long long x = (unsigned long long)key * 0x9E3779B97F4A7C15ULL;
  return x ^ (x >> 32);
}
__device__ __forceinline__ bool bloom_contains(const unsigned long long* bloom, unsigned long long mask,
                                               unsigned long long h) {
  return ((__ldg(bloom + (h & mask)) >> (h & 63)) & 1ULL) && ((__ldg(bloom + ((h >> 17) & mask)) >> ((h >> 6) & 63)) & 1ULL);
}

// Key-hash partition of a join key (the partitioned build's, host side:
// join_partition_of in wg_join.cu).
__host__ __device__ __forceinline__ uint32_t join_partition(long long key, int shift) {
  return (uint32_t)(((unsigned long long)key * 0x9E3779B97F4A7C15ULL) >> shift);
}

// Whether a probe row takes part in this pass of a partitioned build.
__device__ __forceinline__ bool join_pass_mine(const JoinView& j, bool null, long long key) {
  if (j.part_shift == 0) return true;
  if (null) return j.part_lo == 0;
  const uint32_t p = join_partition(key, j.part_shift);
  return p >= (uint32_t)j.part_lo && p < (uint32_t)j.part_hi;
}

// Direct-payload lookup: the payload's raw 32 bits of `key`, or false.
__device__ __forceinline__ bool join_direct(const JoinView& j, int64_t key, int32_t& out, int32_t* err) {
  const unsigned long long* s = (const unsigned long long*)j.slots;
  if (j.dense == 2) {
    const unsigned long long i = (unsigned long long)(key - j.base);
    if (i >= j.mask) return false;
    out = (int32_t)__ldg((const uint32_t*)j.slots + i);
    return true;
  }
  if (j.dense) {
    const unsigned long long i = (unsigned long long)(key - j.base);
    if (i >= j.mask) return false;
    const unsigned long long v = __ldg(s + i);
    if ((uint32_t)v != (uint32_t)(int32_t)key) return false;  // an empty slot holds the sentinel key
    out = (int32_t)(v >> 32);
    return true;
  }
  if (key < INT32_MIN || key > INT32_MAX || key == (int64_t)j.sentinel) return false;
  const uint32_t k32 = (uint32_t)(int32_t)key;
  uint64_t h = fib_slot((uint64_t)key, j.shift);
  for (uint64_t probe = 0; probe <= j.mask; ++probe) {
    const unsigned long long v = __ldg(s + h);
    if ((uint32_t)v == k32) { out = (int32_t)(v >> 32); return true; }
    if ((int32_t)(uint32_t)v == j.sentinel) return false;
    h = (h + 1) & j.mask;
  }
  set_error(err, WG_DERR_TABLE_FULL);
  return false;
}

// join_direct for an int32 probe key: the dense index in 32-bit arithmetic.
// A slot holds the key base + index, and every build key is an int32, so an
// index that wrapped around 2^32 lies past the last key and fails the bound.
__device__ __forceinline__ bool join_direct_i32(const JoinView& j, int32_t key, int32_t& out, int32_t* err) {
  if (!j.dense) return join_direct(j, (int64_t)key, out, err);
  const uint32_t i = (uint32_t)key - (uint32_t)j.base;
  if (i >= (uint32_t)j.mask) return false;  // mask = key span <= 2^30
  if (j.dense == 2) {
    const uint32_t* p = (const uint32_t*)j.slots + i;
    out = (int32_t)(j.l2keep ? ld_keep_u32(p) : __ldg(p));
    return true;
  }
  const unsigned long long* q = (const unsigned long long*)j.slots + i;
  const unsigned long long v = j.l2keep ? ld_keep_u64(q) : __ldg(q);
  if ((uint32_t)v != (uint32_t)key) return false;
  out = (int32_t)(v >> 32);
  return true;
}

// Chain head of `key`, or -1 when absent (HashJoinProbe's idx.Get, join.go:2700).
__device__ __forceinline__ int32_t join_head(const JoinView& j, int64_t key, int32_t* err) {
  if (j.bloom != nullptr && !bloom_contains(j.bloom, j.bloom_mask, bloom_hash_int(key))) return -1;
  uint64_t h = fib_slot((uint64_t)key, j.shift);
  if (j.flavor == 0) {
    if (key < INT32_MIN || key > INT32_MAX) return -1;
    const unsigned long long* s = (const unsigned long long*)j.slots;
    const uint32_t k32 = (uint32_t)(int32_t)key;
    for (uint64_t probe = 0; probe <= j.mask; ++probe) {
      unsigned long long v = __ldg(s + h);
      int32_t head = (int32_t)(v >> 32);
      if (head == -1) return -1;
      if ((uint32_t)v == k32) return head;
      h = (h + 1) & j.mask;
    }
  } else {
    const longlong2* s = (const longlong2*)j.slots;
    for (uint64_t probe = 0; probe <= j.mask; ++probe) {
      longlong2 v = __ldg(s + h);
      int32_t head = (int32_t)(uint32_t)v.y;
      if (head == -1) return -1;
      if (v.x == key) return head;
      h = (h + 1) & j.mask;
    }
  }
  set_error(err, WG_DERR_TABLE_FULL);
  return -1;
}

}  // namespace wgd
