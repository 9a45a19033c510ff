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
//           CTA (the scatter's offsets) and per (first, second)-level bucket;
//  scatter1 the rows passing the filters, as the columns the aggregate reads
//           (keys and aggregate inputs, projections evaluated), written in
//           first-level order (top b1 bits of the key hash);
//  scatter2 each first-level partition re-partitioned by the next b2 hash
//           bits, so every bucket's rows are contiguous;
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

constexpr size_t hc_count_smem(int np1, int nb) { return (size_t)np1 * 4 + (size_t)nb * 4; }

// Rows passing the filters per first-level partition seen by each CTA
// (counts1[p * gridDim.x + cta]) and per bucket over the whole input
// (hist[p1 << b2 | p2], accumulated across calls).
__global__ void __launch_bounds__(kPartThreads) hc_count_kernel(const __grid_constant__ Plan P, int b1, int b2,
                                                                uint32_t* counts1, unsigned long long* hist) {
  extern __shared__ uint32_t hsm[];
  const int np1 = 1 << b1, nb = 1 << (b1 + b2);
  uint32_t* h1 = hsm;
  uint32_t* h2 = hsm + np1;
  for (int i = threadIdx.x; i < np1 + nb; i += blockDim.x) hsm[i] = 0;
  __syncthreads();
  const DynShape sh{P};
  for (int64_t t0 = (int64_t)blockIdx.x * kPartTile; t0 < P.n_items; t0 += (int64_t)gridDim.x * kPartTile) {
    const int m = (int)min((int64_t)kPartTile, P.n_items - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      if (!row_passes(P, sh, t0 + k)) continue;
      const unsigned long long h = row_key_hash(P, sh, t0 + k);
      atomicAdd(&h1[(uint32_t)(h >> (64 - b1))], 1u);
      atomicAdd(&h2[(uint32_t)(h >> (64 - b1 - b2))], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < np1; i += blockDim.x) counts1[(size_t)i * gridDim.x + blockIdx.x] = h1[i];
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    if (h2[i]) atomicAdd(&hist[i], (unsigned long long)h2[i]);
}

// The columns of the partitioned copy: value of plan virtual column vcol[j],
// es[j] bytes per row.
struct HcCols {
  char* data[WG_MAX_IN];
  int32_t vcol[WG_MAX_IN];
  int32_t es[WG_MAX_IN];
  int32_t n;
};

__device__ __forceinline__ void store_val(char* d, int es, const Val& v) {
  if (es == 4) *(uint32_t*)d = (uint32_t)v.lo;
  else if (es == 8) *(unsigned long long*)d = v.lo;
  else { longlong2 x; x.x = (long long)v.hi; x.y = (long long)v.lo; *(longlong2*)d = x; }  // {hi, lo}
}

__host__ __device__ constexpr size_t hc_scatter_smem(int np) {
  return (size_t)np * 8 + (size_t)np * 12 + (size_t)kPartTile * 4;
}

// First level: the input's rows passing the filters, written as the copy's
// columns in partition order (partition p of CTA c from offs[p * gridDim.x + c];
// tiles as hc_count_kernel). Per tile the rows are counting-sorted by
// partition in shared memory and written column by column in that order.
__global__ void __launch_bounds__(kPartThreads) hc_scatter1_kernel(const __grid_constant__ Plan P, int b1,
                                                                   const unsigned long long* offs,
                                                                   const __grid_constant__ HcCols out) {
  extern __shared__ unsigned long long gcur[];
  __shared__ uint32_t warp_tot[32];
  const int np = 1 << b1;
  uint32_t* hist = (uint32_t*)(gcur + np);
  uint32_t* loff = hist + np;
  uint32_t* lcur = loff + np;
  uint16_t* part = (uint16_t*)(lcur + np);      // partition of tile row k (np = dropped)
  uint16_t* perm = part + kPartTile;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    gcur[i] = offs[(size_t)i * gridDim.x + blockIdx.x];
    hist[i] = 0;
  }
  __syncthreads();
  const DynShape sh{P};
  for (int64_t t0 = (int64_t)blockIdx.x * kPartTile; t0 < P.n_items; t0 += (int64_t)gridDim.x * kPartTile) {
    const int m = (int)min((int64_t)kPartTile, P.n_items - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      uint32_t p = (uint32_t)np;
      if (row_passes(P, sh, t0 + k)) {
        p = (uint32_t)(row_key_hash(P, sh, t0 + k) >> (64 - b1));
        atomicAdd(&hist[p], 1u);
      }
      part[k] = (uint16_t)p;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += blockDim.x) { loff[i] = hist[i]; lcur[i] = 0; }
    __syncthreads();
    block_exclusive_scan(loff, np, warp_tot);
    uint32_t kept = 0;  // rows of the tile that pass (loff[np - 1] + hist[np - 1])
    kept = loff[np - 1] + hist[np - 1];
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const uint32_t p = part[k];
      if (p < (uint32_t)np) perm[loff[p] + atomicAdd(&lcur[p], 1u)] = (uint16_t)k;
    }
    __syncthreads();
    for (int j = 0; j < out.n; ++j) {
      const int es = out.es[j];
      char* dcol = out.data[j];
      if (out.vcol[j] < P.n_in) {  // an input column: its bytes as they are
        const char* scol = (const char*)P.in[out.vcol[j]].data + t0 * es;
        for (uint32_t q = threadIdx.x; q < kept; q += blockDim.x) {
          const int k = perm[q];
          const uint32_t p = part[k];
          char* d = dcol + (gcur[p] + (q - loff[p])) * es;
          const char* sp = scol + (size_t)k * es;
          if (es == 4) *(uint32_t*)d = __ldg((const uint32_t*)sp);
          else if (es == 8) *(unsigned long long*)d = __ldg((const unsigned long long*)sp);
          else *(longlong2*)d = __ldg((const longlong2*)sp);
        }
        continue;
      }
      for (uint32_t q = threadIdx.x; q < kept; q += blockDim.x) {  // a projection, evaluated per row
        const int k = perm[q];
        const uint32_t p = part[k];
        const SrcGlobal src{t0 + k};
        ExprVals ev;
        eval_exprs(P, sh, src, -1, ev);
        const Val v = fetch(P, sh, src, out.vcol[j], -1, ev);
        store_val(dcol + (gcur[p] + (q - loff[p])) * es, es, v);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += blockDim.x) { gcur[i] += hist[i]; hist[i] = 0; }
    __syncthreads();
  }
}

// Second level, over the copy (plan Pc: its columns are the copy's, no filters
// or projections). Work item w is tile (w - item0[p]) of first-level partition
// p (rows [off1[p], off1[p + 1]) of the copy); its rows go to the buckets
// p << b2 | p2 of the second copy, each tile claiming its rows of a bucket
// with one atomic on the bucket's cursor.
__global__ void __launch_bounds__(kPartThreads) hc_scatter2_kernel(const __grid_constant__ Plan Pc, int b1, int b2,
                                                                   const int64_t* off1, const int64_t* item0,
                                                                   int np1, int64_t n_items_total,
                                                                   unsigned long long* cursor,
                                                                   const __grid_constant__ HcCols out) {
  extern __shared__ unsigned long long base[];  // np2 claimed starts, then the arrays below
  __shared__ uint32_t warp_tot[32];
  __shared__ int s_p;
  const int np2 = 1 << b2;
  uint32_t* hist = (uint32_t*)(base + np2);
  uint32_t* loff = hist + np2;
  uint32_t* lcur = loff + np2;
  uint16_t* part = (uint16_t*)(lcur + np2);
  uint16_t* perm = part + kPartTile;
  const DynShape sh{Pc};
  for (int64_t w = blockIdx.x; w < n_items_total; w += gridDim.x) {
    if (threadIdx.x == 0) {  // the partition holding item w
      int lo = 0, hi = np1 - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (item0[mid] <= w) lo = mid; else hi = mid - 1;
      }
      s_p = lo;
    }
    for (int i = threadIdx.x; i < np2; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const int p = s_p;
    const int64_t t0 = off1[p] + (w - item0[p]) * kPartTile;
    const int m = (int)min((int64_t)kPartTile, off1[p + 1] - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const uint32_t q = (uint32_t)(row_key_hash(Pc, sh, t0 + k) >> (64 - b1 - b2)) & (uint32_t)(np2 - 1);
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
    __syncthreads();
    for (int j = 0; j < out.n; ++j) {
      const int es = out.es[j];
      const char* scol = (const char*)Pc.in[j].data;
      char* dcol = out.data[j];
      for (int qi = threadIdx.x; qi < m; qi += blockDim.x) {
        const int k = perm[qi];
        const uint32_t q = part[k];
        char* d = dcol + (base[q] + (qi - loff[q])) * es;
        const char* sp = scol + (t0 + k) * es;
        if (es == 4) *(uint32_t*)d = __ldg((const uint32_t*)sp);
        else if (es == 8) *(unsigned long long*)d = __ldg((const unsigned long long*)sp);
        else *(longlong2*)d = __ldg((const longlong2*)sp);
      }
    }
    __syncthreads();
  }
}

// Buckets: persistent CTAs take buckets b, b + gridDim.x, ...; bucket b's rows
// are [boff[b], boff[b + 1]) of the plan's columns (the second copy). Each
// bucket is aggregated in the shared table (P.smem_slots slots, P.smem_sw
// words each, slot from the hash bits below the bucket's), new groups that no
// longer fit going to the HBM table P.T; then its groups are appended to
// `out` (P.L.slot_words words each, float-SUM copies folded in) from a cursor
// claimed with one atomic. A result that would pass out_cap rows raises
// *out_over and writes nothing past it.
template <int NA, class Sh>
__global__ void __launch_bounds__(1024, 1) hc_bucket_kernel(const __grid_constant__ Plan P, const int64_t* boff,
                                                            int64_t nb, unsigned long long* out,
                                                            unsigned long long* out_cursor, int64_t out_cap,
                                                            int32_t* out_over) {
  extern __shared__ __align__(16) unsigned long long sm[];
  __shared__ int s_groups;
  __shared__ uint32_t warp_tot[32];
  __shared__ unsigned long long s_base;
  const Sh sh{P};
  Credit cr;
  const int S = P.smem_slots;
  const int s_limit = (S * 7) / 8;
  const int sw = P.L.slot_words, ssw = smem_stride(P), rep = smem_copies(P);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
    smem_table_init(P, sm, S, &s_groups);
    __syncthreads();
    const int64_t r0 = boff[b], r1 = boff[b + 1];
    for (int64_t base = r0 + (int64_t)wid * 32; base < r1; base += (int64_t)nw * 32) {
      const int64_t row = base + lane;
      const bool act = row < r1;
      const SrcGlobal src{act ? row : r0};
      process_rows<NA, true>(P, sh, src, act, sm, &s_groups, s_limit, cr);
    }
    __syncthreads();
    // this thread's used slots: i = threadIdx.x + k * blockDim.x
    uint32_t mine = 0;
    for (int i = threadIdx.x; i < S; i += blockDim.x) mine += sm[(size_t)i * ssw] != P.L.init[0] ||
                                                             (P.L.key_words == 2 && sm[(size_t)i * ssw + 1] != P.L.init[1]);
    uint32_t x = mine;  // exclusive scan of `mine` over the CTA
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(WG_FULL_MASK, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t z = lane < nw ? warp_tot[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(WG_FULL_MASK, z, o);
        if (lane >= o) z += y;
      }
      if (lane < nw) warp_tot[lane] = z;
      if (lane == nw - 1) s_base = z ? atomicAdd(out_cursor, (unsigned long long)z) : 0ULL;
    }
    __syncthreads();
    unsigned long long at = s_base + (wid > 0 ? warp_tot[wid - 1] : 0u) + x - mine;
    for (int i = threadIdx.x; i < S; i += blockDim.x) {
      const unsigned long long* s = sm + (size_t)i * ssw;
      const bool used = s[0] != P.L.init[0] || (P.L.key_words == 2 && s[1] != P.L.init[1]);
      if (!used) continue;
      if ((int64_t)at >= out_cap) { *out_over = 1; ++at; continue; }
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
      ++at;
    }
    __syncthreads();  // the table is re-initialised for the next bucket
  }
  cr.release(P.T);
}

}  // namespace wgd
