// wg_hc.cuh — GROUP BY over far more groups than fit on chip: a two-level
// key-hash partition of the rows in HBM, then every bucket of the second level
// aggregated in one CTA's shared memory.
//
// A table of tens of millions of groups lives in HBM, where each row's update
// is a read-modify-write of a random line (the direct path) or, with the rows
// first grouped by the table region they touch, an L2 atomic per aggregate
// word — and L2 atomics top out near 190 G/s on this part (a 16 MB region, one
// 64-bit add each), about five per row here. Shared-memory atomics run four
// times faster, so the rows are bucketed until one bucket's groups fit one SM:
//
//  count    one pass over the key columns: rows per first-level partition per
//           CTA (the scatter's offsets) and a distinct-key sketch, from which
//           finalize picks b2 (the second level's bits, at most 8) so buckets
//           hold about half a shared table of groups;
//  scatter1 the rows passing the filters, as the columns the aggregate reads
//           (keys and aggregate inputs, projections evaluated), written in
//           first-level order (top b1 bits of the key hash), with a byte per
//           row holding the next 8 hash bits;
//  count2   rows per (partition, bucket), from the top b2 bits of the bytes;
//  scatter2 each first-level partition re-partitioned by its bucket bytes, so
//           every bucket's rows are contiguous;
//  buckets  persistent CTAs take buckets; each aggregates its bucket in a
//           shared-memory table (slots picked by the hash bits below the
//           bucket's) and appends its groups, in the table's slot layout, to a
//           compact result with one atomic per bucket.
//
// A bucket whose groups outgrow the shared table sends its later new groups
// to an HBM table instead (a group lives in exactly one of the two), which
// finalize appends to the result.
#pragma once

#include "wg_shapes.cuh"

namespace wgd {

// The 64-bit key hash the partitions and buckets split on: fib_slot's product
// for one key word, packed_slot's for two (NULL keys hash to 0; the mode
// refuses inputs with validity bitmaps, so none reach here).
template <class Sh>
__device__ __forceinline__ unsigned long long row_key_hash(const Plan& P, const Sh& sh, int64_t row) {
  const SrcGlobal src{row};
  ExprVals ev;
  eval_exprs(P, sh, src, -1, ev);
  unsigned long long k0 = 0, k1 = 0;
  bool knull = false;
  make_key(P, sh, src, -1, ev, k0, k1, knull);
  if (knull) return 0ULL;
  if (sh.key_words() == 1) return k0 * 0x9E3779B97F4A7C15ULL;
  const unsigned long long a = k0 ^ 0x9E3779B97F4A7C15ULL, b = k1 ^ 0x517CC1B727220A95ULL;
  return (__umul64hi(a, b) ^ (a * b) ^ (k0 + k1)) * 0x9E3779B97F4A7C15ULL;
}

template <class Sh>
__device__ __forceinline__ bool row_passes(const Plan& P, const Sh& sh, int64_t row) {
  const SrcGlobal src{row};
#pragma unroll
  for (int f = 0; f < WG_MAX_FILTERS; ++f) {
    if (f >= sh.n_filters()) break;
    if (!pred_val(P, sh, f, src.in(P, sh, sh.filt_col(f)))) return false;
  }
  return true;
}

// The count and the first-level scatter walk the input in tiles of TILE
// rows, CTA c taking tiles c, c + gridDim.x, ... (both launched on the same
// grid, one 1024-thread CTA per SM), so the rows a CTA counts per partition
// are exactly the rows it later writes there.
// Tiles of TILE rows, 8 per thread: 8192-row tiles in one 1024-thread CTA per
// SM, or 4096-row tiles in two 512-thread CTAs per SM (WG_HC_TILE), whose
// phases then overlap.
constexpr int kHcThreads = 1024;  // count2's CTAs
template <int TILE> struct HcGeom {
  static_assert(TILE == 8192 || TILE == 4096, "tile rows");
  static constexpr int threads = TILE / 8;
  static constexpr int ctas = 8192 / TILE;  // per SM
  static constexpr int stage_bytes = TILE * 16;  // one column of up to 16-byte values
};

// Bits of the per-row bucket byte the first level writes: the second level
// uses its top b2 <= 8 bits, b2 chosen when the groups have been estimated.
constexpr int kHcByteBits = 8;
// Distinct-key sketch of the counting pass: 2^kHllBits registers, each the
// largest rank (leading zeros + 1) among the hashes that select it.
constexpr int kHllBits = 10;
constexpr size_t hc_count_smem(int np1) { return (size_t)np1 * 4 + ((size_t)1 << kHllBits) * 4; }

// Rows passing the filters per first-level partition seen by each CTA
// (counts1[p * gridDim.x + cta]), and the distinct-key sketch of those rows
// (max-merged into hll). Register index: the hash's low kHllBits bits; rank:
// leading zeros of the remaining bits, plus one. The low bits are independent
// of the top bits that pick partitions and buckets.
template <int TILE, class Sh>
__global__ void __launch_bounds__(HcGeom<TILE>::threads, HcGeom<TILE>::ctas) hc_count_kernel(const __grid_constant__ Plan P, int b1,
                                                                 uint32_t* counts1, uint32_t* hll) {
  extern __shared__ uint32_t h1[];
  const int np1 = 1 << b1;
  uint32_t* reg = h1 + np1;
  for (int i = threadIdx.x; i < np1 + (1 << kHllBits); i += blockDim.x) h1[i] = 0;
  __syncthreads();
  const Sh sh{P};
  for (int64_t t0 = (int64_t)blockIdx.x * TILE; t0 < P.n_items; t0 += (int64_t)gridDim.x * TILE) {
    const int m = (int)min((int64_t)TILE, P.n_items - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      if (!row_passes(P, sh, t0 + k)) continue;
      const unsigned long long h = row_key_hash(P, sh, t0 + k);
      atomicAdd(&h1[(uint32_t)(h >> (64 - b1))], 1u);
      const uint32_t rank = (uint32_t)(__clzll((long long)((h >> kHllBits) | 1ULL)) - kHllBits + 1);
      const uint32_t r = (uint32_t)h & ((1u << kHllBits) - 1u);
      if (rank > reg[r]) atomicMax(&reg[r], rank);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < np1; i += blockDim.x) counts1[(size_t)i * gridDim.x + blockIdx.x] = h1[i];
  for (int i = threadIdx.x; i < (1 << kHllBits); i += blockDim.x)
    if (reg[i]) atomicMax(&hll[i], reg[i]);
}

// The columns of the partitioned copy: value of plan virtual column vcol[j],
// es[j] bytes per row.
struct HcCols {
  char* data[WG_MAX_IN];
  int32_t vcol[WG_MAX_IN];
  int32_t es[WG_MAX_IN];
  int32_t n;
};

// Shared memory of the scatter kernels: the staging area, np output cursors
// (8 B) and per-partition hist / offset / cursor (12 B), then per tile row its
// partition and its place in the order (2 B each) and, for the first level,
// its bucket byte. One CTA per SM.
__host__ __device__ constexpr size_t hc_scatter_smem(int tile, int np, bool bucket_bytes) {
  return (size_t)tile * 16 + (size_t)np * 20 + (size_t)tile * (bucket_bytes ? 5 : 4);
}

// A column value as the copy stores it: 4 or 8 bytes in x, a 16-byte one as
// {x = hi, y = lo}.
__device__ __forceinline__ ulonglong2 copy_val(int es, const Val& v) {
  ulonglong2 r;
  r.x = es == 16 ? v.hi : v.lo;
  r.y = v.lo;
  return r;
}

// Row r of input column j read as it lies (es bytes).
__device__ __forceinline__ ulonglong2 hc_raw(const Plan& P, int j, int es, int64_t r) {
  const char* base = (const char*)P.in[j].data;
  ulonglong2 v;
  v.y = 0;
  if (es == 4) {
    v.x = __ldg((const uint32_t*)base + r);
  } else if (es == 8) {
    v.x = __ldg((const unsigned long long*)base + r);
  } else {
    const longlong2 t = __ldg((const longlong2*)base + r);
    v.x = (unsigned long long)t.x;
    v.y = (unsigned long long)t.y;
  }
  return v;
}

__device__ __forceinline__ void stage_put(void* stage, int es, int k, ulonglong2 v) {
  if (es == 4) ((uint32_t*)stage)[k] = (uint32_t)v.x;
  else if (es == 8) ((unsigned long long*)stage)[k] = v.x;
  else ((ulonglong2*)stage)[k] = v;
}

// Tile rows in partition order. Position q of the order holds tile row
// perm[q] of partition part[perm[q]], which goes to output row
// dst[p] + q - loff[p]. The column's tile values are in `stage` in tile-row
// order (staged with coalesced reads); they are stored in partition order
// (stores in runs of one partition).
__device__ __forceinline__ void hc_store_column(const void* stage, uint32_t kept, const uint16_t* perm,
                                                const uint16_t* part, const unsigned long long* dst,
                                                const uint32_t* loff, char* dcol, int es) {
  for (uint32_t q = threadIdx.x; q < kept; q += blockDim.x) {
    const int k = perm[q];
    const uint32_t p = part[k];
    const unsigned long long row = dst[p] + (q - loff[p]);
    if (es == 4) ((uint32_t*)dcol)[row] = ((const uint32_t*)stage)[k];
    else if (es == 8) ((unsigned long long*)dcol)[row] = ((const unsigned long long*)stage)[k];
    else ((ulonglong2*)dcol)[row] = ((const ulonglong2*)stage)[k];
  }
}

// First level: the input's rows passing the filters, written as the copy's
// columns in partition order (partition p of CTA c from offs[p * gridDim.x + c];
// tiles as hc_count_kernel), and with each row its bucket byte (the next 8
// hash bits), from which the second level splits without hashing again.
// Every input byte is read from HBM once: the first n_pre copy columns (input
// key columns of 4 or 8 bytes) are staged side by side while the rows are
// hashed, the other columns one at a time afterwards.
template <int TILE, class Sh>
__global__ void __launch_bounds__(HcGeom<TILE>::threads, HcGeom<TILE>::ctas) hc_scatter1_kernel(const __grid_constant__ Plan P, int b1,
                                                                    const unsigned long long* offs,
                                                                    const __grid_constant__ HcCols out, int n_pre,
                                                                    uint8_t* bucket_out) {
  extern __shared__ __align__(16) unsigned long long stage[];
  __shared__ uint32_t warp_tot[32];
  __shared__ int pre_off[WG_MAX_IN];
  const int np = 1 << b1;
  char* stg = (char*)stage;
  unsigned long long* gcur = (unsigned long long*)(stg + HcGeom<TILE>::stage_bytes);
  uint32_t* hist = (uint32_t*)(gcur + np);
  uint32_t* loff = hist + np;
  uint32_t* lcur = loff + np;
  uint16_t* part = (uint16_t*)(lcur + np);  // partition of tile row k (np = dropped)
  uint16_t* perm = part + TILE;
  uint8_t* bkt = (uint8_t*)(perm + TILE);
  if (threadIdx.x == 0) {
    int off = 0;
    for (int j = 0; j < n_pre; ++j) { pre_off[j] = off; off += TILE * out.es[j]; }
  }
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    gcur[i] = offs[(size_t)i * gridDim.x + blockIdx.x];
    hist[i] = 0;
  }
  __syncthreads();
  const Sh sh{P};
  for (int64_t t0 = (int64_t)blockIdx.x * TILE; t0 < P.n_items; t0 += (int64_t)gridDim.x * TILE) {
    const int m = (int)min((int64_t)TILE, P.n_items - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      uint32_t p = (uint32_t)np;
      for (int j = 0; j < n_pre; ++j)
        stage_put(stg + pre_off[j], out.es[j], k, hc_raw(P, out.vcol[j], out.es[j], t0 + k));
      if (row_passes(P, sh, t0 + k)) {
        const unsigned long long h = row_key_hash(P, sh, t0 + k);
        p = (uint32_t)(h >> (64 - b1));
        bkt[k] = (uint8_t)(h >> (64 - b1 - kHcByteBits));
        atomicAdd(&hist[p], 1u);
      }
      part[k] = (uint16_t)p;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += blockDim.x) { loff[i] = hist[i]; lcur[i] = 0; }
    __syncthreads();
    block_exclusive_scan(loff, np, warp_tot);
    const uint32_t kept = loff[np - 1] + hist[np - 1];  // rows of the tile that pass
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const uint32_t p = part[k];
      if (p < (uint32_t)np) perm[loff[p] + atomicAdd(&lcur[p], 1u)] = (uint16_t)k;
    }
    __syncthreads();
    for (int j = 0; j < n_pre; ++j)  // staged while hashing
      hc_store_column(stg + pre_off[j], kept, perm, part, gcur, loff, out.data[j], out.es[j]);
    for (uint32_t q = threadIdx.x; q < kept; q += blockDim.x) {
      const int k = perm[q];
      const uint32_t p = part[k];
      bucket_out[gcur[p] + (q - loff[p])] = bkt[k];
    }
    for (int j = n_pre; j < out.n; ++j) {
      const int es = out.es[j], vc = out.vcol[j];
      __syncthreads();  // the staging area is free again
      if (vc < P.n_in) {  // an input column: its bytes as they are
#pragma unroll 4
        for (int k = threadIdx.x; k < m; k += blockDim.x) stage_put(stg, es, k, hc_raw(P, vc, es, t0 + k));
      } else {  // a projection, evaluated per kept row
        for (int k = threadIdx.x; k < m; k += blockDim.x) {
          if (part[k] >= (uint16_t)np) continue;
          const SrcGlobal src{t0 + k};
          ExprVals ev;
          eval_exprs(P, sh, src, -1, ev);
          stage_put(stg, es, k, copy_val(es, fetch(P, sh, src, vc, -1, ev)));
        }
      }
      __syncthreads();
      hc_store_column(stg, kept, perm, part, gcur, loff, out.data[j], es);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += blockDim.x) { gcur[i] += hist[i]; hist[i] = 0; }
    __syncthreads();
  }
}

// A run's partition starts and first work items, copied to shared memory once
// per CTA (np1 <= 256).
struct HcRunIndex {
  int64_t off1[257];
  int64_t item0[257];
};
__device__ __forceinline__ void hc_load_index(HcRunIndex& ix, const int64_t* off1, const int64_t* item0, int np1) {
  for (int i = threadIdx.x; i <= np1; i += blockDim.x) {
    ix.off1[i] = off1[i];
    ix.item0[i] = item0[i];
  }
  __syncthreads();
}

// The partition holding work item w (item0: first item of each partition).
__device__ __forceinline__ int hc_item_partition(const int64_t* item0, int np1, int64_t w) {
  int lo = 0, hi = np1 - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (item0[mid] <= w) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Rows per bucket of a first-level run: work item w is tile (w - item0[p]) of
// partition p (rows [off1[p], off1[p + 1]) of the run); bucket q of the
// partition is the top b2 bits of the row's byte; hist[p << b2 | q]
// accumulates across runs.
template <int TILE>
__global__ void __launch_bounds__(kHcThreads) hc_count2_kernel(const uint8_t* bucket, int b2, const int64_t* off1,
                                                               const int64_t* item0, int np1, int64_t n_items_total,
                                                               unsigned long long* hist) {
  __shared__ uint32_t h[256];
  __shared__ HcRunIndex ix;
  const int np2 = 1 << b2;
  hc_load_index(ix, off1, item0, np1);
  for (int64_t w = blockIdx.x; w < n_items_total; w += gridDim.x) {
    for (int i = threadIdx.x; i < np2; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int p = hc_item_partition(ix.item0, np1, w);
    const int64_t t0 = ix.off1[p] + (w - ix.item0[p]) * TILE;
    const int m = (int)min((int64_t)TILE, ix.off1[p + 1] - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) atomicAdd(&h[bucket[t0 + k] >> (kHcByteBits - b2)], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < np2; i += blockDim.x)
      if (h[i]) atomicAdd(&hist[((size_t)p << b2) | (size_t)i], (unsigned long long)h[i]);
    __syncthreads();
  }
}

// Second level, over a run (plan Pc: its columns are the copy's, no filters or
// projections), items as hc_count2_kernel; each tile's rows go to the buckets
// p << b2 | q of the second copy, the tile claiming its rows of a bucket
// with one atomic on the bucket's cursor.
template <int TILE>
__global__ void __launch_bounds__(HcGeom<TILE>::threads, HcGeom<TILE>::ctas) hc_scatter2_kernel(const __grid_constant__ Plan Pc, int b2,
                                                                    const uint8_t* bucket, const int64_t* off1,
                                                                    const int64_t* item0, int np1,
                                                                    int64_t n_items_total, unsigned long long* cursor,
                                                                    const __grid_constant__ HcCols out) {
  extern __shared__ __align__(16) unsigned long long stage[];
  __shared__ uint32_t warp_tot[32];
  __shared__ HcRunIndex ix;
  const int np2 = 1 << b2;
  char* stg = (char*)stage;
  unsigned long long* base = (unsigned long long*)(stg + HcGeom<TILE>::stage_bytes);
  uint32_t* hist = (uint32_t*)(base + np2);
  uint32_t* loff = hist + np2;
  uint32_t* lcur = loff + np2;
  uint16_t* part = (uint16_t*)(lcur + np2);
  uint16_t* perm = part + TILE;
  hc_load_index(ix, off1, item0, np1);
  for (int64_t w = blockIdx.x; w < n_items_total; w += gridDim.x) {
    for (int i = threadIdx.x; i < np2; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const int p = hc_item_partition(ix.item0, np1, w);
    const int64_t t0 = ix.off1[p] + (w - ix.item0[p]) * TILE;
    const int m = (int)min((int64_t)TILE, ix.off1[p + 1] - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const uint32_t q = (uint32_t)bucket[t0 + k] >> (kHcByteBits - b2);
      part[k] = (uint16_t)q;
      atomicAdd(&hist[q], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np2; i += blockDim.x) {
      loff[i] = hist[i];
      lcur[i] = 0;
      base[i] = hist[i] ? atomicAdd(&cursor[((size_t)p << b2) | (size_t)i], (unsigned long long)hist[i]) : 0ULL;
    }
    __syncthreads();
    block_exclusive_scan(loff, np2, warp_tot);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const uint32_t q = part[k];
      perm[loff[q] + atomicAdd(&lcur[q], 1u)] = (uint16_t)k;
    }
    for (int j = 0; j < out.n; ++j) {
      const int es = out.es[j];
      __syncthreads();  // perm complete; the staging area free again
#pragma unroll 4
      for (int k = threadIdx.x; k < m; k += blockDim.x) stage_put(stg, es, k, hc_raw(Pc, j, es, t0 + k));
      __syncthreads();
      hc_store_column(stg, (uint32_t)m, perm, part, base, loff, out.data[j], es);
    }
    __syncthreads();
  }
}

// Buckets: persistent CTAs (1024 / THREADS per SM, each with its share of the
// SM's shared memory) take buckets b, b + gridDim.x, ...; bucket b's rows are
// [boff[b], boff[b + 1]) of the plan's columns (the second copy). Each bucket
// is aggregated in the shared table (P.smem_slots slots of P.smem_sw words,
// slot from the hash bits below the bucket's; new groups that no longer fit go
// to the HBM table P.T). Each insert appends its slot to the used-slot list
// (P.smem_list), so a bucket's groups are appended to `out` (P.L.slot_words
// words each, float-SUM copies folded in, from a cursor claimed with one
// atomic) and their slots re-initialised without sweeping the whole table,
// which is initialised once. A result that would pass out_cap rows raises
// *out_over and writes nothing past it.
template <int NA, class Sh, int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) hc_bucket_kernel(const __grid_constant__ Plan P,
                                                                            const int64_t* boff, int64_t nb,
                                                                            unsigned long long* out,
                                                                            unsigned long long* out_cursor,
                                                                            int64_t out_cap, int32_t* out_over) {
  extern __shared__ __align__(16) unsigned long long sm[];
  __shared__ int s_groups;
  __shared__ unsigned long long s_base;
  const Sh sh{P};
  Credit cr;
  const int S = P.smem_slots;
  const int s_limit = (S * 7) / 8;
  const int sw = P.L.slot_words, ssw = smem_stride(P), rep = smem_copies(P);
  const uint32_t* list = (const uint32_t*)(sm + P.smem_list);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  smem_table_init(P, sm, S, &s_groups);
  __syncthreads();
  for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const int64_t r0 = boff[b], r1 = boff[b + 1];
    for (int64_t base = r0 + (int64_t)wid * 32; base < r1; base += (int64_t)nw * 32) {
      const int64_t row = base + lane;
      const bool act = row < r1;
      const SrcGlobal src{act ? row : r0};
      process_rows<NA, true>(P, sh, src, act, sm, &s_groups, s_limit, cr);
    }
    __syncthreads();
    const int ng = min(s_groups, S);
    if (threadIdx.x == 0) s_base = ng ? atomicAdd(out_cursor, (unsigned long long)ng) : 0ULL;
    __syncthreads();
    for (int i = threadIdx.x; i < ng; i += blockDim.x) {
      unsigned long long* s = sm + (size_t)list[i] * ssw;
      const unsigned long long at = s_base + (unsigned long long)i;
      if ((int64_t)at >= out_cap) {
        *out_over = 1;
      } else {
        unsigned long long* d = out + at * (unsigned long long)sw;
        for (int w = 0; w < sw; ++w) d[w] = s[w];
        int nf = 0;
        for (int a = 0; a < P.L.n_aggs; ++a) {
          if (P.L.agg[a].kind != K_SUM_F64) continue;
          double t = as_f(s[P.L.agg[a].off]);
          for (int r = 1; r < rep; ++r) t = __dadd_rn(t, as_f(s[sw + nf * (rep - 1) + (r - 1)]));
          d[P.L.agg[a].off] = as_w(t);
          ++nf;
        }
      }
      for (int w = 0; w < ssw; ++w) s[w] = w < sw ? P.L.init[w] : 0ULL;  // empty again for the next bucket
    }
    if (threadIdx.x == 0) s_groups = 0;
    __syncthreads();
  }
  cr.release(P.T);
}

}  // namespace wgd
