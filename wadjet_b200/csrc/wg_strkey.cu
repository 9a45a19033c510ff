// wg_strkey.cu — string GROUP BY keys: a device dictionary from each distinct
// string to a dense group id.
//
// The reference groups one STRING / BYTES column through strHashTable
// (consumeBatchStrGroup, exec/aggregate.go:3038): a string's bytes are the
// key, a NULL string has its own group. Here a consume call first maps every
// row's string to a dense int32 id in a dictionary that lives with the
// aggregate, then aggregates over the ids like any int key (the NULL rows keep
// the string column's validity, so they form the NULL-key group); an export
// or emit reports ids, and wg_agg_key_strings turns ids back into strings.
//
// The dictionary is an open-addressing table of 128-bit key hashes installed
// with one 16-byte compare-and-swap, plus an arena holding each distinct
// string once. Per batch: (1) a hash pass writes every row's hash and sketches
// the batch's distinct strings, the table is sized from the sketch and every
// row finds or installs its hash, each install listing its slot; (2) in the
// same pass the rows of a slot with no id yet elect its lowest row; (3) the
// list, sorted by those rows, gives each new string its id in first-appearance
// order and (by a scan of the lengths) its arena offset, and the elected row
// copies the bytes; (4) every row compares its bytes with its string's arena
// copy and takes the id. A 128-bit collision between two different strings
// would make (4) fail, which the call reports instead of merging the groups.
// No step waits on another thread.
#include "wg_internal.h"
#include "wg_device.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

using namespace wgd;

constexpr unsigned long long kEmpty = ~0ULL;
constexpr uint32_t kNoRep = 0xFFFFFFFFu;
constexpr unsigned long long kNoId = ~0ULL;  // a slot whose string has no id yet
constexpr int kLenShift = 40;  // slot / id location: arena offset | length << 40

struct StrSrc {
  const uint32_t* offs;
  const uint8_t* bytes;
  const uint64_t* valid;  // the column's validity words (nullptr: no NULLs)
  const uint32_t* sel;    // selection entries (nullptr: rows 0 .. n - 1)
  int64_t n;              // items
};

__device__ __forceinline__ int64_t item_row(const StrSrc& s, int64_t i) { return s.sel ? (int64_t)s.sel[i] : i; }

__device__ __forceinline__ bool row_null(const StrSrc& s, int64_t row) {
  return s.valid != nullptr && ((s.valid[row >> 6] >> (row & 63)) & 1ULL) == 0;
}

// k (1..8) bytes at p as a little-endian word, zero above them. Only aligned
// 8-byte words holding at least one of the k bytes are read, so no read leaves
// the pages the string lies in.
__device__ __forceinline__ unsigned long long load_bytes8(const uint8_t* p, uint32_t k) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const unsigned long long* w = reinterpret_cast<const unsigned long long*>(a & ~uintptr_t(7));
  const uint32_t sh = (uint32_t)(a & 7);
  unsigned long long v = __ldg(w) >> (sh * 8);
  if (sh + k > 8) v |= __ldg(w + 1) << ((8 - sh) * 8);
  return k >= 8 ? v : (v & ((1ULL << (k * 8)) - 1));
}

// MurmurHash3's 64-bit finalizer (Appleby, public domain).
__device__ __forceinline__ unsigned long long fmix64(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// Two 64-bit hashes of a string, eight bytes a step: a multiply-rotate and a
// multiply-xorshift chain over the words, each finished with the length and
// fmix64. Neither word is ~0, so {~0, ~0} stays the empty slot.
__device__ __forceinline__ U128 str_hash(const uint8_t* p, uint32_t n) {
  unsigned long long a = 0x9E3779B97F4A7C15ULL ^ (unsigned long long)n, b = 0xC2B2AE3D27D4EB4FULL + n;
  for (uint32_t j = 0; j < n; j += 8) {
    const unsigned long long c = load_bytes8(p + j, min(8u, n - j));
    a = (a ^ c) * 0x87C37B91114253D5ULL;
    a = (a << 31) | (a >> 33);
    b = (b + c) * 0x4CF5AD432745937FULL;
    b ^= b >> 29;
  }
  U128 h;
  h.lo = fmix64(a ^ ((unsigned long long)n << 32));
  h.hi = fmix64(b + a);
  if (h.lo == kEmpty) h.lo = kEmpty - 1;
  if (h.hi == kEmpty) h.hi = kEmpty - 1;
  return h;
}

// The n bytes at p and q are equal (eight at a time).
__device__ __forceinline__ bool bytes_equal(const uint8_t* p, const uint8_t* q, uint32_t n) {
  for (uint32_t j = 0; j < n; j += 8) {
    const uint32_t k = min(8u, n - j);
    if (load_bytes8(p + j, k) != load_bytes8(q + j, k)) return false;
  }
  return true;
}

// Append `v` for the lanes with `mine` set to list[ctr[2]...], one atomic per
// warp. Every lane of the warp calls it together.
__device__ __forceinline__ void warp_append(bool mine, uint32_t v, uint32_t* list, unsigned long long* count) {
  const unsigned m = __ballot_sync(0xFFFFFFFFu, mine);
  if (m == 0) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(m));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  if (mine) list[base + __popc(m & ((1u << lane) - 1u))] = v;
}

// Distinct-hash sketch of a batch (HyperLogLog, Flajolet, Fusy, Gandouet and
// Meunier 2007): 2^kSketchBits registers, each the largest rank (leading zeros
// + 1) of the hashes that fall in it. It sizes the table before the insert
// pass, so a batch of many new strings does not fill a small table first.
constexpr int kSketchBits = 10;
constexpr int kProbeLimit = 4096;  // an insert probing further asks for a larger table

// (1a) Each item's 128-bit hash ({~0, ~0} for a NULL string) and the sketch.
__global__ void str_hash_kernel(StrSrc s, U128* hashes, uint32_t* sketch) {
  __shared__ uint32_t reg[1 << kSketchBits];
  for (int r = threadIdx.x; r < (1 << kSketchBits); r += blockDim.x) reg[r] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = item_row(s, i);
    U128 k;
    if (row_null(s, row)) {
      k.lo = kEmpty;
      k.hi = kEmpty;
    } else {
      const uint32_t b0 = s.offs[row];
      k = str_hash(s.bytes + b0, s.offs[row + 1] - b0);
      const uint32_t r = (uint32_t)(k.hi >> (64 - kSketchBits));
      const uint32_t rank = (uint32_t)__clzll((long long)((k.hi << kSketchBits) | (1ULL << (kSketchBits - 1)))) + 1;
      if (reg[r] < rank) atomicMax(reg + r, rank);
    }
    hashes[i] = k;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < (1 << kSketchBits); r += blockDim.x)
    if (reg[r] != 0) atomicMax(sketch + r, reg[r]);
}

// (1b) Find or install each non-NULL item's hash: rowslot[i] = its slot, -1 for
// a NULL string, -2 when the probe passed kProbeLimit slots (ctr[1] is then
// raised and the host grows the table and runs the pass again). ctr[0] counts
// the installs (added once per CTA); each install appends its slot to `list`
// (ctr[2] counts them). (2) The items of a slot with no id yet elect the
// lowest of them (rep).
__global__ void str_insert_kernel(const U128* hashes, int64_t n, unsigned long long* slots, uint64_t mask,
                                  int32_t* rowslot, uint32_t* rep, uint32_t* list, unsigned long long* ctr) {
  __shared__ unsigned int installs;
  if (threadIdx.x == 0) installs = 0;
  __syncthreads();
  const uint64_t limit = mask < (uint64_t)kProbeLimit ? mask + 1 : (uint64_t)kProbeLimit;
  // the loop's trip count is the same for every lane of a warp (warp_append)
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    bool installed = false;
    int32_t found = -1;
    if (i < n) {
      const U128 k = hashes[i];
      if (!(k.lo == kEmpty && k.hi == kEmpty)) {
        uint64_t idx = (k.lo ^ (k.lo >> 32)) & mask;
        found = -2;
        for (uint64_t probe = 0; probe < limit; ++probe) {
          unsigned long long* sl = slots + idx * 4;
          const U128 cur = read128(sl);
          if (cur.lo == k.lo && cur.hi == k.hi) { found = (int32_t)idx; break; }
          if (cur.lo == kEmpty || cur.hi == kEmpty) {  // empty, or a key being installed
            U128 e; e.lo = kEmpty; e.hi = kEmpty;
            const U128 old = cas128((U128*)sl, e, k);
            if (old.lo == e.lo && old.hi == e.hi) {
              installed = true;
              found = (int32_t)idx;
              break;
            }
            if (old.lo == k.lo && old.hi == k.hi) { found = (int32_t)idx; break; }
          }
          idx = (idx + 1) & mask;
        }
        if (found == -2) {
          ctr[1] = 1;
        } else if (slots[(int64_t)found * 4 + 2] == kNoId && *(volatile uint32_t*)(rep + found) > (uint32_t)i) {
          // a string new in this batch: its lowest item represents it (the
          // atomic only when it can lower the candidate, so a frequent
          // string's rows do not all hit one word)
          atomicMin(rep + found, (uint32_t)i);
        }
      }
      rowslot[i] = found;
    }
    if (installed) atomicAdd(&installs, 1u);
    warp_append(installed, (uint32_t)found, list, ctr + 2);
  }
  __syncthreads();
  if (threadIdx.x == 0 && installs != 0) atomicAdd(ctr, (unsigned long long)installs);
}

// (3) Sort keys of the strings new in this batch: the slot above its
// representative item, so sorting by the low bits gives first-appearance order.
__global__ void str_key_kernel(const uint32_t* list, int64_t k, const uint32_t* rep, unsigned long long* keys) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < k; t += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t sl = list[t];
    keys[t] = ((unsigned long long)sl << 32) | rep[sl];
  }
}

// The new strings' total length (the last length plus the last offset).
__global__ void str_bytes_kernel(const unsigned long long* lens, const unsigned long long* pre, int64_t k,
                                 unsigned long long* ctr) {
  ctr[3] = lens[k - 1] + pre[k - 1];
}

// (4a) The length of each new string, in first-appearance order (keys sorted).
__global__ void str_len_kernel(StrSrc s, const unsigned long long* keys, int64_t k, unsigned long long* lens) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < k; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = item_row(s, (int64_t)(keys[t] & 0xFFFFFFFFULL));
    lens[t] = s.offs[row + 1] - s.offs[row];
  }
}

// (4b) The t-th new string (by first appearance) takes id id0 + t and its
// bytes go to the arena at off0 + pre[t].
__global__ void str_assign_kernel(StrSrc s, const unsigned long long* keys, int64_t k, const unsigned long long* pre,
                                  unsigned long long* slots, uint32_t* rep, unsigned long long id0,
                                  unsigned long long off0, uint8_t* arena, unsigned long long* id_loc) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < k; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = (int64_t)(keys[t] & 0xFFFFFFFFULL);
    const uint32_t sl = (uint32_t)(keys[t] >> 32);
    const int64_t row = item_row(s, i);
    const uint32_t b0 = s.offs[row], len = s.offs[row + 1] - b0;
    const unsigned long long off = off0 + pre[t];
    for (uint32_t q = 0; q < len; ++q) arena[off + q] = s.bytes[b0 + q];
    const unsigned long long loc = off | ((unsigned long long)len << kLenShift);
    id_loc[id0 + t] = loc;
    slots[(int64_t)sl * 4 + 3] = loc;
    slots[(int64_t)sl * 4 + 2] = id0 + t;
    rep[sl] = kNoRep;
  }
}

// (5) Every item checks its bytes against its string's arena copy and takes
// the id (ids are indexed by row; rows outside the selection are not written;
// a NULL string's row gets 0 under its NULL bit).
__global__ void str_gid_kernel(StrSrc s, const unsigned long long* slots, const int32_t* rowslot,
                               const uint8_t* arena, int32_t* gid, int32_t* err) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = item_row(s, i);
    const int32_t sl = rowslot[i];
    if (sl < 0) { gid[row] = 0; continue; }
    const unsigned long long loc = __ldg(slots + (int64_t)sl * 4 + 3);
    const uint32_t len = (uint32_t)(loc >> kLenShift);
    const uint32_t b0 = s.offs[row], n = s.offs[row + 1] - b0;
    if (n != len || !bytes_equal(s.bytes + b0, arena + (loc & ((1ULL << kLenShift) - 1)), n))
      set_error(err, WG_DERR_HASH_COLLISION);
    gid[row] = (int32_t)__ldg(slots + (int64_t)sl * 4 + 2);
  }
}

// The dictionary's slots moved into a larger table.
// (The table grown between insert passes.) The old slots move to the new
// table; those installed by the stopped pass (no id yet) are listed again at
// their new places.
__global__ void str_rehash_kernel(const unsigned long long* old, uint64_t old_cap, unsigned long long* slots,
                                  uint64_t mask, uint32_t* list, unsigned long long* count) {
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < old_cap; i0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = i0 + threadIdx.x;
    bool pending = false;
    uint32_t at = 0;
    if (i < old_cap) {
      const unsigned long long* o = old + i * 4;
      if (!(o[0] == kEmpty && o[1] == kEmpty)) {
        U128 k; k.lo = o[0]; k.hi = o[1];
        uint64_t idx = (k.lo ^ (k.lo >> 32)) & mask;
        for (uint64_t probe = 0; probe <= mask; ++probe) {
          unsigned long long* sl = slots + idx * 4;
          U128 e; e.lo = kEmpty; e.hi = kEmpty;
          const U128 prev = cas128((U128*)sl, e, k);
          if (prev.lo == e.lo && prev.hi == e.hi) {
            sl[2] = o[2];
            sl[3] = o[3];
            pending = o[2] == kNoId;
            at = (uint32_t)idx;
            break;
          }
          idx = (idx + 1) & mask;
        }
      }
    }
    warp_append(pending, at, list, count);
  }
}

__global__ void str_init_slots_kernel(unsigned long long* slots, uint64_t cap) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x) {
    slots[i * 4] = kEmpty;
    slots[i * 4 + 1] = kEmpty;
    slots[i * 4 + 2] = kNoId;
    slots[i * 4 + 3] = 0;
  }
}

// ctr[0] = the slots in use, ctr[1] = 0 (not full), ctr[2..3] = 0 (new strings, their bytes)
__global__ void str_ctr_kernel(unsigned long long* ctr, unsigned long long used) {
  ctr[0] = used;
  ctr[1] = 0;
  ctr[2] = 0;
  ctr[3] = 0;
}

}  // namespace

namespace wg {

struct StrDict {
  DevBuf slots, rep, ctr, arena, id_loc;
  uint64_t cap = 0;                 // table slots (a power of two)
  int64_t n_ids = 0, used = 0;      // distinct strings and arena bytes
  int64_t slots_used = 0;           // installed hashes (n_ids after every complete batch)
  DevBuf hashes, sketch, rowslot, list, sorted, pack, pre, scan_tmp, gid;  // per-batch scratch
  bool dirty = false;               // a batch stopped part way: refused until reset
  DevBuf h_offs, h_bytes, h_valid, h_sel;             // a host batch's string column on the device
  std::vector<unsigned long long> loc_host;           // host copies for wg_agg_key_strings,
  std::vector<uint8_t> arena_host;                    // valid while no batch came since
  bool host_fresh = false;
};

namespace {

unsigned str_grid(Ctx* ctx, int64_t n, int block) {
  const int64_t want = (n + block - 1) / block;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)ctx->sm_count * 16));
}

// Grow a device buffer to `need` bytes, keeping its first `keep` bytes.
wg_status grow_keep(Ctx* ctx, DevBuf& b, int64_t keep, int64_t need) {
  if (b.bytes() >= need) return WG_OK;
  DevBuf nb;
  WG_TRY(nb.alloc(ctx, std::max<int64_t>(need, b.bytes() * 2)));
  if (keep > 0) WG_CUDA_TRY(cudaMemcpyAsync(nb.get(), b.get(), (size_t)keep, cudaMemcpyDeviceToDevice, ctx->stream));
  b = std::move(nb);  // the old buffer's cudaFree waits for the copy
  return WG_OK;
}

// A table of `cap` slots holding the old table's strings.
wg_status str_table(Ctx* ctx, StrDict* d, uint64_t cap) {
  DevBuf ns, nr;
  WG_TRY(ns.alloc(ctx, (int64_t)cap * 32));
  WG_TRY(nr.alloc(ctx, (int64_t)cap * 4));
  str_init_slots_kernel<<<str_grid(ctx, (int64_t)cap, 256), 256, 0, ctx->stream>>>(ns.as<unsigned long long>(), cap);
  ctx->count_launch();
  WG_CUDA_TRY(cudaMemsetAsync(nr.get(), 0xFF, (size_t)cap * 4, ctx->stream));
  if (d->cap > 0) {
    str_rehash_kernel<<<str_grid(ctx, (int64_t)d->cap, 256), 256, 0, ctx->stream>>>(
        d->slots.as<unsigned long long>(), d->cap, ns.as<unsigned long long>(), cap - 1, d->list.as<uint32_t>(),
        d->ctr.as<unsigned long long>() + 2);
    ctx->count_launch();
  }
  WG_CUDA_TRY(cudaGetLastError());
  d->slots = std::move(ns);
  d->rep = std::move(nr);
  d->cap = cap;
  return WG_OK;
}

// The sketch's distinct-count estimate: the harmonic-mean estimator with the
// linear-counting correction for small counts (Flajolet et al. 2007).
wg_status sketch_estimate(Ctx* ctx, StrDict* d, double* out) {
  const int m = 1 << kSketchBits;
  uint32_t reg[1 << kSketchBits];
  WG_CUDA_TRY(cudaMemcpyAsync(reg, d->sketch.get(), sizeof(reg), cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  double z = 0.0;
  int zeros = 0;
  for (int r = 0; r < m; ++r) { z += std::ldexp(1.0, -(int)reg[r]); zeros += reg[r] == 0; }
  double e = 0.7213 / (1.0 + 1.079 / m) * m * m / z;
  if (e <= 2.5 * m && zeros > 0) e = m * std::log((double)m / zeros);
  *out = e;
  return WG_OK;
}

uint64_t pow2_at_least(uint64_t v) {
  uint64_t c = 1024;
  while (c < v) c <<= 1;
  return c;
}

}  // namespace

void strdict_free(StrDict* d) { delete d; }

// Forget every string; the buffers (and the table's size) stay for the next query.
void strdict_reset(StrDict* d, Ctx* ctx) {
  if (!d) return;
  if (d->cap > 0) {
    str_init_slots_kernel<<<str_grid(ctx, (int64_t)d->cap, 256), 256, 0, ctx->stream>>>(d->slots.as<unsigned long long>(),
                                                                                    d->cap);
    ctx->count_launch();
    cudaMemsetAsync(d->rep.get(), 0xFF, (size_t)d->cap * 4, ctx->stream);
  }
  d->n_ids = 0; d->used = 0; d->slots_used = 0; d->dirty = false;
  d->loc_host.clear(); d->arena_host.clear(); d->host_fresh = false;
}

int64_t strdict_size(const StrDict* d) { return d ? d->n_ids : 0; }


wg_status strdict_map(Ctx* ctx, StrDict** dp, const wg_batch_desc* in, int col, bool host, int64_t hint,
                      wg_column* out) {
  const wg_column& c = in->cols[col];
  const wg_bytes* sb = static_cast<const wg_bytes*>(c.data);
  const int64_t len = in->len;
  if (!sb || (len > 0 && (!sb->offsets || !sb->bytes))) return fail(WG_E_INVALID, "string column without offsets or bytes");
  if (len >= (int64_t)INT32_MAX) return fail(WG_E_UNSUPPORTED, "a string-keyed batch holds fewer than 2^31 rows");
  if (in->sel && in->sel_len > len) return fail(WG_E_INVALID, "selection longer than the batch");
  if (!*dp) *dp = new StrDict();
  StrDict* d = *dp;
  if (d->dirty) return fail(WG_E_STATE, "the string dictionary stopped part way through a batch; reset the aggregate");
  d->host_fresh = false;
  const int64_t n = in->sel ? in->sel_len : len;
  StrSrc s{sb->offsets, sb->bytes, c.valid_words, in->sel, n};
  if (host) {
    // the string column (and the selection) on the device; the other columns
    // are staged by the caller
    const int64_t total = len > 0 ? (int64_t)sb->offsets[len] : 0;
    WG_TRY(d->h_offs.ensure(ctx, std::max<int64_t>((len + 1) * 4, 16)));
    WG_TRY(d->h_bytes.ensure(ctx, std::max<int64_t>(total, 16)));
    if (len > 0)
      WG_CUDA_TRY(cudaMemcpyAsync(d->h_offs.get(), sb->offsets, (size_t)(len + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (total > 0)
      WG_CUDA_TRY(cudaMemcpyAsync(d->h_bytes.get(), sb->bytes, (size_t)total, cudaMemcpyHostToDevice, ctx->stream));
    s.offs = d->h_offs.as<uint32_t>();
    s.bytes = d->h_bytes.as<uint8_t>();
    if (c.valid_words) {
      const int64_t words = (len + 63) / 64;
      WG_TRY(d->h_valid.ensure(ctx, std::max<int64_t>(words * 8, 16)));
      if (words > 0)
        WG_CUDA_TRY(cudaMemcpyAsync(d->h_valid.get(), c.valid_words, (size_t)words * 8, cudaMemcpyHostToDevice, ctx->stream));
      s.valid = d->h_valid.as<uint64_t>();
    }
    if (in->sel) {
      WG_TRY(d->h_sel.ensure(ctx, std::max<int64_t>(n * 4, 16)));
      if (n > 0) WG_CUDA_TRY(cudaMemcpyAsync(d->h_sel.get(), in->sel, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
      s.sel = d->h_sel.as<uint32_t>();
    }
  }
  WG_TRY(d->gid.ensure(ctx, std::max<int64_t>(len * 4, 16)));
  *out = wg_column{WG_TYPE_INT32, 0, d->gid.get(), s.valid, len};
  if (n == 0) return WG_OK;

  // (1) hash every item and sketch the batch's distinct strings; size the
  // table for the strings so far plus the sketch's estimate (load at most 2/3
  // when the estimate holds), then install the hashes, growing the table and
  // running the pass again if a probe ran long
  WG_TRY(d->hashes.ensure(ctx, n * 16));
  WG_TRY(d->sketch.ensure(ctx, (int64_t(1) << kSketchBits) * 4));
  WG_TRY(d->rowslot.ensure(ctx, n * 4));
  WG_TRY(d->list.ensure(ctx, std::max<int64_t>(n * 4, 16)));
  WG_TRY(d->ctr.ensure(ctx, 64));
  unsigned long long* ctr = d->ctr.as<unsigned long long>();
  const unsigned grid = str_grid(ctx, n, 256);
  WG_CUDA_TRY(cudaMemsetAsync(d->sketch.get(), 0, (size_t(1) << kSketchBits) * 4, ctx->stream));
  str_hash_kernel<<<grid, 256, 0, ctx->stream>>>(s, d->hashes.as<U128>(), d->sketch.as<uint32_t>());
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  double est = 0.0;
  WG_TRY(sketch_estimate(ctx, d, &est));
  d->dirty = true;  // until the batch completes
  str_ctr_kernel<<<1, 1, 0, ctx->stream>>>(ctr, (unsigned long long)d->slots_used);
  ctx->count_launch();
  const uint64_t want = pow2_at_least((uint64_t)(1.5 * ((double)d->slots_used + std::min<double>((double)n, est * 1.1)) + 64));
  if (d->cap < want) WG_TRY(str_table(ctx, d, want));
  int64_t cv[4] = {0, 0, 0, 0};
  for (int pass = 0;; ++pass) {
    str_insert_kernel<<<grid, 256, 0, ctx->stream>>>(d->hashes.as<U128>(), n, d->slots.as<unsigned long long>(),
                                                     d->cap - 1, d->rowslot.as<int32_t>(), d->rep.as<uint32_t>(),
                                                     d->list.as<uint32_t>(), ctr);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    WG_TRY(read_back_i64(ctx, reinterpret_cast<int64_t*>(ctr), cv, 3));
    if (cv[1] == 0) break;
    if (pass >= 16 || d->cap >= (1ULL << 31)) return fail(WG_E_NOMEM, "string dictionary table cannot grow");
    // the installs of the stopped pass stay in the table; the grown table's
    // rehash lists them again, the next pass lists its own installs
    d->slots_used = cv[0];
    str_ctr_kernel<<<1, 1, 0, ctx->stream>>>(ctr, (unsigned long long)d->slots_used);
    ctx->count_launch();
    WG_TRY(str_table(ctx, d, std::max<uint64_t>(d->cap * 4, pow2_at_least(2 * (uint64_t)cv[0]))));
  }
  d->slots_used = cv[0];
  const int64_t new_ids = cv[2];
  if (d->n_ids + new_ids >= (int64_t)INT32_MAX) return fail(WG_E_UNSUPPORTED, "more than 2^31 - 1 distinct strings");

  int64_t new_bytes = 0;
  if (new_ids > 0) {
    // (3)-(4) the new strings in first-appearance order (sorted by their first
    // item), ids and arena offsets from a scan of their lengths
    WG_TRY(d->pack.ensure(ctx, new_ids * 8));     // sort keys, then lengths
    WG_TRY(d->sorted.ensure(ctx, new_ids * 8));   // sorted keys
    WG_TRY(d->pre.ensure(ctx, new_ids * 8));
    int bits = 1;
    while (bits < 32 && (int64_t(1) << bits) < n) ++bits;
    size_t t1 = 0, t2 = 0;
    WG_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, t1, d->pack.as<unsigned long long>(),
                                               d->sorted.as<unsigned long long>(), (int)new_ids, 0, bits, ctx->stream));
    WG_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, t2, d->pack.as<unsigned long long>(),
                                              d->pre.as<unsigned long long>(), (int)new_ids, ctx->stream));
    WG_TRY(d->scan_tmp.ensure(ctx, std::max<int64_t>((int64_t)std::max(t1, t2), 16)));
    const unsigned kgrid = str_grid(ctx, new_ids, 256);
    str_key_kernel<<<kgrid, 256, 0, ctx->stream>>>(d->list.as<uint32_t>(), new_ids, d->rep.as<uint32_t>(),
                                                   d->pack.as<unsigned long long>());
    WG_CUDA_TRY(cub::DeviceRadixSort::SortKeys(d->scan_tmp.get(), t1, d->pack.as<unsigned long long>(),
                                               d->sorted.as<unsigned long long>(), (int)new_ids, 0, bits, ctx->stream));
    str_len_kernel<<<kgrid, 256, 0, ctx->stream>>>(s, d->sorted.as<unsigned long long>(), new_ids,
                                                   d->pack.as<unsigned long long>());
    WG_CUDA_TRY(cub::DeviceScan::ExclusiveSum(d->scan_tmp.get(), t2, d->pack.as<unsigned long long>(),
                                              d->pre.as<unsigned long long>(), (int)new_ids, ctx->stream));
    str_bytes_kernel<<<1, 1, 0, ctx->stream>>>(d->pack.as<unsigned long long>(), d->pre.as<unsigned long long>(),
                                               new_ids, ctr);
    ctx->count_launch(3 + 2 + 2);  // key, lengths, total; the sort's and the scan's kernels (about two each)
    WG_CUDA_TRY(cudaGetLastError());
    WG_TRY(read_back_i64(ctx, reinterpret_cast<int64_t*>(ctr), cv, 4));
    new_bytes = cv[3];
    WG_TRY(grow_keep(ctx, d->arena, d->used, std::max<int64_t>(d->used + new_bytes, 16)));
    WG_TRY(grow_keep(ctx, d->id_loc, d->n_ids * 8, std::max<int64_t>((d->n_ids + new_ids) * 8, 16)));
    str_assign_kernel<<<kgrid, 256, 0, ctx->stream>>>(s, d->sorted.as<unsigned long long>(), new_ids,
                                                      d->pre.as<unsigned long long>(), d->slots.as<unsigned long long>(),
                                                      d->rep.as<uint32_t>(), (unsigned long long)d->n_ids,
                                                      (unsigned long long)d->used, d->arena.as<uint8_t>(),
                                                      d->id_loc.as<unsigned long long>());
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
  }
  // (5) every item's bytes checked against its string's arena copy, and its id
  str_gid_kernel<<<grid, 256, 0, ctx->stream>>>(s, d->slots.as<unsigned long long>(), d->rowslot.as<int32_t>(),
                                                d->arena.as<uint8_t>(), d->gid.as<int32_t>(), ctx->dev_error);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  d->n_ids += new_ids;
  d->used += new_bytes;
  d->dirty = false;
  return check_device_error(ctx);
}

wg_status strdict_strings(Ctx* ctx, StrDict* d, const int64_t* ids, int64_t n, uint32_t* out_offsets,
                          uint8_t* out_bytes, int64_t bytes_cap, int64_t* need_bytes) {
  const int64_t n_ids = d ? d->n_ids : 0;
  if (d && !d->host_fresh) {
    d->loc_host.resize((size_t)n_ids);
    d->arena_host.resize((size_t)d->used);
    if (n_ids > 0)
      WG_CUDA_TRY(cudaMemcpyAsync(d->loc_host.data(), d->id_loc.get(), (size_t)n_ids * 8, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    if (d->used > 0)
      WG_CUDA_TRY(cudaMemcpyAsync(d->arena_host.data(), d->arena.get(), (size_t)d->used, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    d->host_fresh = true;
  }
  int64_t total = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (ids[i] < 0 || ids[i] >= n_ids) return fail(WG_E_INVALID, "string id out of range");
    total += (int64_t)(d->loc_host[(size_t)ids[i]] >> kLenShift);
  }
  if (total > (int64_t)UINT32_MAX) return fail(WG_E_UNSUPPORTED, "strings longer than 32-bit offsets reach");
  *need_bytes = total;
  if (total > bytes_cap) return WG_OK;
  int64_t pos = 0;
  out_offsets[0] = 0;
  for (int64_t i = 0; i < n; ++i) {
    const unsigned long long loc = d->loc_host[(size_t)ids[i]];
    const int64_t len = (int64_t)(loc >> kLenShift), off = (int64_t)(loc & ((1ULL << kLenShift) - 1));
    if (len > 0) std::memcpy(out_bytes + pos, d->arena_host.data() + off, (size_t)len);
    pos += len;
    out_offsets[i + 1] = (uint32_t)pos;
  }
  return WG_OK;
}

}  // namespace wg
