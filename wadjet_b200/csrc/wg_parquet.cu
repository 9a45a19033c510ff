// wg_parquet.cu — batches on the device: the upload of decoded host batches and
// Parquet column chunks decoded on the GPU.
//
// The reference's native scan decodes each page on the host
// (ColumnPageReader.decodeValues, internal/storage/parquet/page_reader.go:607;
// the RLE / bit-packed hybrid, rle.go) and copies the values into a
// batch.Vector (scan/columnar_native.go:470-707). Here only the encoded page
// bytes cross to the device and the decode runs there:
//
//  1. definition levels (one CTA per page): the hybrid stream expanded to a
//     valid byte per row (level 1 = a value, 0 = NULL);
//  2. the bytes packed into validity words, their popcounts scanned, so the
//     rank of a row among the non-NULL rows is a prefix plus one popcount;
//  3. values (one CTA per page): PLAIN values copied, or dictionary indices
//     expanded from the hybrid stream and gathered from the dictionary with
//     the reference's bounds check, each widened on the way (DECIMAL's INT64
//     to Int128 as Int128From); a chunk without NULLs writes the column
//     directly, otherwise the non-NULL values go to a dense buffer and
//  4. scatter to their rows by rank.
//
// The hybrid run headers are varints, so one thread per CTA walks them (up to
// kRuns at a time into shared memory) and the whole CTA expands those runs in
// parallel; pages decode side by side on different SMs.
#include "wg_internal.h"
#include "wg_device.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <climits>

using namespace wg;

struct wg_batch {
  wg::Ctx* ctx = nullptr;
  std::vector<wg::DevBuf> data, valid;
  wg::DevBuf sel;
  std::vector<wg_column> cols;
  int64_t len = 0, sel_len = 0;
  bool has_sel = false;
};

namespace {

using namespace wgd;

constexpr int kPageThreads = 512;
constexpr int kRuns = 256;

struct PageD {
  int64_t row0, n;            // the page's rows within the chunk
  int64_t def_off, def_len;   // level bytes in the chunk's byte buffer (def_len < 0: no levels)
  int64_t data_off, data_len; // values section in the chunk's byte buffer
  int32_t enc;
  int32_t _pad;
};

struct Run {
  int64_t out0, n;    // values [out0, out0 + n) of the stream
  int64_t off, blen;  // bit-packed: the run's bytes
  int32_t kind;       // 0 = repeated value, 1 = bit-packed
  int32_t value;
};

// Value j of a bit-packed run whose bytes are p[0, blen): the reference reads
// up to four little-endian bytes from the value's first byte, bytes past the
// run's end reading as zero, and masks bit_width bits (decodeBitPackedRange,
// rle.go:214-250).
__device__ __forceinline__ int32_t bitpacked_value(const uint8_t* p, int64_t blen, int bw, int64_t j) {
  if (bw == 0) return 0;
  const int64_t bit = j * bw;
  const int64_t byte = bit >> 3;
  const int sh = (int)(bit & 7);
  uint32_t raw = 0;
  const int64_t rem = blen - byte;
  for (int i = 0; i < 4; ++i)
    if (i < rem) raw |= (uint32_t)p[byte + i] << (8 * i);
  const int32_t mask = bw >= 32 ? -1 : (int32_t)((1u << bw) - 1u);
  return (int32_t)(raw >> sh) & mask;
}

// The RLE / bit-packed hybrid stream p[0, len) with bit width bw, up to
// `count` values, handed to sink(k, value) for k = 0, 1, ... (decodeAllBatch,
// rle.go:219-275). Every thread of the CTA calls it; it returns the number of
// values decoded (fewer than count when the stream ends early). A varint that
// runs off the stream or a repeated value missing its bytes sets
// WG_DERR_BAD_PAGE, as the reference returns an error there.
template <class Sink>
__device__ int64_t hybrid_decode(const uint8_t* p, int64_t len, int bw, int64_t count, Sink& sink, int32_t* err) {
  __shared__ Run runs[kRuns];
  __shared__ int s_nruns, s_done;
  __shared__ long long s_off, s_pos, s_next;
  if (threadIdx.x == 0) { s_off = 0; s_pos = 0; }
  __syncthreads();
  const int vbytes = (bw + 7) / 8;
  for (;;) {
    if (threadIdx.x == 0) {
      int nr = 0, done = 0;
      int64_t off = s_off, pos = s_pos;
      while (nr < kRuns) {
        if (off >= len || pos >= count) { done = 1; break; }
        unsigned long long h = 0;
        int shift = 0;
        bool ok = false;
        while (off < len && shift < 64) {
          const uint8_t b = p[off++];
          h |= (unsigned long long)(b & 0x7F) << shift;
          if (!(b & 0x80)) { ok = true; break; }
          shift += 7;
        }
        if (!ok) { set_error(err, WG_DERR_BAD_PAGE); done = 1; break; }
        if ((h & 1ULL) == 0) {  // repeated value: count = header >> 1, then ceil(bw/8) value bytes
          const int64_t c = (int64_t)(h >> 1);
          if (off + vbytes > len) { set_error(err, WG_DERR_BAD_PAGE); done = 1; break; }
          int32_t v = 0;
          for (int i = 0; i < vbytes; ++i) v |= (int32_t)p[off + i] << (8 * i);
          off += vbytes;
          const int64_t n = c < count - pos ? c : count - pos;
          if (n > 0) { runs[nr].out0 = pos; runs[nr].n = n; runs[nr].off = 0; runs[nr].blen = 0; runs[nr].kind = 0; runs[nr].value = v; ++nr; }
          pos += n;
        } else {  // bit-packed: header >> 1 groups of 8 values, groups * bw bytes
          const int64_t groups = (int64_t)(h >> 1);
          if (groups <= 0) continue;
          if (groups > LLONG_MAX / 8 || (bw > 0 && groups > LLONG_MAX / bw)) {
            set_error(err, WG_DERR_BAD_PAGE); done = 1; break;
          }
          const int64_t nv = groups * 8;
          const int64_t n = nv < count - pos ? nv : count - pos;
          int64_t bc = groups * bw;
          if (off + bc > len) bc = len - off;
          runs[nr].out0 = pos; runs[nr].n = n; runs[nr].off = off; runs[nr].blen = bc; runs[nr].kind = 1; runs[nr].value = 0;
          ++nr;
          off += bc;
          pos += n;
        }
      }
      s_nruns = nr;
      s_done = done;
      s_off = off;
      s_next = pos;
    }
    __syncthreads();
    const int nr = s_nruns;
    if (nr > 0) {
      const int64_t base = runs[0].out0, total = (int64_t)s_next - base;
      for (int64_t k = threadIdx.x; k < total; k += blockDim.x) {
        const int64_t o = base + k;
        int lo = 0, hi = nr - 1;  // the last run starting at or before o
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (runs[mid].out0 <= o) lo = mid; else hi = mid - 1;
        }
        const Run& r = runs[lo];
        const int32_t v = r.kind == 0 ? r.value : bitpacked_value(p + r.off, r.blen, bw, o - r.out0);
        sink(o, v);
      }
    }
    __syncthreads();
    const int done = s_done;
    if (threadIdx.x == 0) s_pos = s_next;
    __syncthreads();
    if (done) break;
  }
  return (int64_t)s_pos;
}

struct ChunkArgs {
  const PageD* pages;
  const uint8_t* bytes;
  int32_t n_pages;
  int32_t es;              // physical width: 4 or 8
  int32_t widen;           // INT64 DECIMAL values to Int128
  int32_t nullable;        // some page has definition levels
  const void* dict;
  int64_t dict_len;
  uint8_t* vbytes;         // valid flag per row of the chunk
  const uint64_t* vwords;  // validity words
  const unsigned long long* wprefix;  // non-NULL rows before each 64-row word (words + 1 entries)
  char* dense;             // non-NULL values in row order (the column itself when nothing is NULL)
  int32_t* err;
  int64_t rows;
};

__device__ __forceinline__ int64_t rank_of(const ChunkArgs& a, int64_t r) {
  if (!a.nullable) return r;
  const int64_t w = r >> 6;
  const int b = (int)(r & 63);
  const uint64_t below = b ? (a.vwords[w] & ((~0ULL) >> (64 - b))) : 0ULL;
  return (int64_t)a.wprefix[w] + __popcll(below);
}

// One physical value (es bytes) stored at output slot i, widened for DECIMAL.
__device__ __forceinline__ void put_value(const ChunkArgs& a, int64_t i, const uint8_t* src) {
  if (a.widen) {
    const long long v = *(const long long*)src;
    longlong2 d;
    d.x = v < 0 ? -1LL : 0LL;  // Int128From: Hi is the sign extension (decimal.go:17)
    d.y = v;
    ((longlong2*)a.dense)[i] = d;
  } else if (a.es == 4) {
    ((uint32_t*)a.dense)[i] = *(const uint32_t*)src;
  } else {
    ((unsigned long long*)a.dense)[i] = *(const unsigned long long*)src;
  }
}

struct DefSink {
  uint8_t* v;
  __device__ __forceinline__ void operator()(int64_t k, int32_t level) const { v[k] = level == 1 ? 1 : 0; }
};

struct DictSink {
  const ChunkArgs* a;
  int64_t dense0;
  __device__ __forceinline__ void operator()(int64_t k, int32_t idx) const {
    // the gather loops' bounds check (columnar_native.go:480-486): uint(idx) >= len is an error
    if ((uint64_t)(uint32_t)idx >= (uint64_t)a->dict_len) { set_error(a->err, WG_DERR_BAD_PAGE); return; }
    put_value(*a, dense0 + k, (const uint8_t*)a->dict + (int64_t)(uint32_t)idx * a->es);
  }
};

__global__ void __launch_bounds__(kPageThreads) def_levels_kernel(const ChunkArgs a) {
  const PageD pg = a.pages[blockIdx.x];
  uint8_t* v = a.vbytes + pg.row0;
  if (pg.def_len < 0) {  // a required page inside a nullable chunk: every row has a value
    for (int64_t k = threadIdx.x; k < pg.n; k += blockDim.x) v[k] = 1;
    return;
  }
  DefSink sink{v};
  const int64_t got = hybrid_decode(a.bytes + pg.def_off, pg.def_len, 1, pg.n, sink, a.err);
  if (threadIdx.x == 0 && got < pg.n) set_error(a.err, WG_DERR_BAD_PAGE);
}

// Validity words and their popcounts from the per-row flags.
__global__ void pack_valid_kernel(const uint8_t* v, int64_t rows, uint64_t* words, unsigned long long* cnt,
                                  int64_t nwords) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (int64_t)gridDim.x * blockDim.x) {
    uint64_t bits = 0;
    const int64_t r0 = w * 64;
    for (int b = 0; b < 64 && r0 + b < rows; ++b) bits |= (uint64_t)(v[r0 + b] != 0) << b;
    words[w] = bits;
    cnt[w] = (unsigned long long)__popcll(bits);
  }
}

__global__ void __launch_bounds__(kPageThreads) values_kernel(const ChunkArgs a) {
  const PageD pg = a.pages[blockIdx.x];
  const int64_t d0 = rank_of(a, pg.row0);
  const int64_t cnt = rank_of(a, pg.row0 + pg.n) - d0;
  const uint8_t* data = a.bytes + pg.data_off;
  if (pg.enc == WG_ENC_PLAIN) {
    if (pg.data_len < cnt * a.es) {  // PLAIN data shorter than the page's values
      if (threadIdx.x == 0) set_error(a.err, WG_DERR_BAD_PAGE);
      return;
    }
    for (int64_t k = threadIdx.x; k < cnt; k += blockDim.x) put_value(a, d0 + k, data + k * a.es);
    return;
  }
  // dictionary indices: one bit-width byte, then the hybrid stream
  if (cnt == 0) return;
  if (pg.data_len < 1 || data[0] > 32) {
    if (threadIdx.x == 0) set_error(a.err, WG_DERR_BAD_PAGE);
    return;
  }
  DictSink sink{&a, d0};
  const int64_t got = hybrid_decode(data + 1, pg.data_len - 1, (int)data[0], cnt, sink, a.err);
  if (threadIdx.x == 0 && got < cnt) set_error(a.err, WG_DERR_BAD_PAGE);  // fewer indices than values
}

// Non-NULL values to their rows; NULL rows get zero bytes.
__global__ void scatter_kernel(const ChunkArgs a, char* out, int out_es) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < a.rows; r += (int64_t)gridDim.x * blockDim.x) {
    const bool valid = (a.vwords[r >> 6] >> (r & 63)) & 1ULL;
    const int64_t k = valid ? rank_of(a, r) : 0;
    if (out_es == 16) {
      longlong2 z; z.x = 0; z.y = 0;
      ((longlong2*)out)[r] = valid ? ((const longlong2*)a.dense)[k] : z;
    } else if (out_es == 8) {
      ((unsigned long long*)out)[r] = valid ? ((const unsigned long long*)a.dense)[k] : 0ULL;
    } else {
      ((uint32_t*)out)[r] = valid ? ((const uint32_t*)a.dense)[k] : 0u;
    }
  }
}

unsigned grid_for_rows(Ctx* ctx, int64_t n, int block) {
  int64_t b = (n + block - 1) / block;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)ctx->sm_count * 16));
}

// Physical width of a column type's PLAIN values (4 or 8), 0 when the GPU path has none.
int64_t phys_width(int32_t type_id) {
  if (type_id == WG_TYPE_DECIMAL) return 8;
  const int64_t e = elem_size(type_id);
  return e == 4 || e == 8 ? e : 0;
}

wg_status decode_chunk(Ctx* ctx, const wg_column_chunk& ch, int64_t rows, DevBuf& out, DevBuf& out_valid,
                       bool* has_valid) {
  const int64_t es = phys_width(ch.type_id);
  const int64_t oes = elem_size(ch.type_id);
  if (es == 0 || oes == 0) return fail(WG_E_UNSUPPORTED, "column type is not on the GPU decode path");
  bool nullable = false, dict_enc = false;
  int64_t bytes = 0;
  for (int p = 0; p < ch.n_pages; ++p) {
    const wg_page& pg = ch.pages[p];
    if (pg.num_values < 0 || pg.def_len < 0 || pg.data_len < 0 || (pg.def_len > 0 && !pg.def_levels) ||
        (pg.data_len > 0 && !pg.data))
      return fail(WG_E_INVALID, "bad page descriptor");
    if (pg.encoding != WG_ENC_PLAIN && pg.encoding != WG_ENC_PLAIN_DICTIONARY && pg.encoding != WG_ENC_RLE_DICTIONARY)
      return fail(WG_E_UNSUPPORTED, "page encoding is not on the GPU decode path (PLAIN and dictionary are)");
    nullable |= pg.def_levels != nullptr;
    dict_enc |= pg.encoding != WG_ENC_PLAIN;
    bytes += ((pg.def_len + 15) & ~int64_t(15)) + ((pg.data_len + 15) & ~int64_t(15));
  }
  if (dict_enc && (!ch.dict || ch.dict_len < 0)) return fail(WG_E_INVALID, "dictionary page missing");
  // one buffer with every page's bytes; the page table; the dictionary
  DevBuf dbytes, dpages, ddict;
  std::vector<PageD> pt((size_t)ch.n_pages);
  std::vector<char> host((size_t)std::max<int64_t>(bytes, 16));
  int64_t at = 0, row = 0;
  for (int p = 0; p < ch.n_pages; ++p) {
    const wg_page& pg = ch.pages[p];
    PageD& d = pt[(size_t)p];
    d.row0 = row;
    d.n = pg.num_values;
    d.enc = pg.encoding;
    d._pad = 0;
    if (pg.def_levels) {
      d.def_off = at;
      d.def_len = pg.def_len;
      std::memcpy(host.data() + at, pg.def_levels, (size_t)pg.def_len);
      at += (pg.def_len + 15) & ~int64_t(15);
    } else {
      d.def_off = 0;
      d.def_len = -1;
    }
    d.data_off = at;
    d.data_len = pg.data_len;
    if (pg.data_len) std::memcpy(host.data() + at, pg.data, (size_t)pg.data_len);
    at += (pg.data_len + 15) & ~int64_t(15);
    row += pg.num_values;
  }
  if (row != rows) return fail(WG_E_INVALID, "column chunks of one batch must hold the same number of rows");
  WG_TRY(dbytes.alloc(ctx, std::max<int64_t>(bytes, 16)));
  WG_TRY(dpages.alloc(ctx, (int64_t)pt.size() * (int64_t)sizeof(PageD) + 16));
  if (bytes) WG_CUDA_TRY(cudaMemcpyAsync(dbytes.get(), host.data(), (size_t)bytes, cudaMemcpyHostToDevice, ctx->stream));
  WG_CUDA_TRY(cudaMemcpyAsync(dpages.get(), pt.data(), pt.size() * sizeof(PageD), cudaMemcpyHostToDevice, ctx->stream));
  if (dict_enc && ch.dict_len > 0) {
    WG_TRY(ddict.alloc(ctx, ch.dict_len * es));
    WG_CUDA_TRY(cudaMemcpyAsync(ddict.get(), ch.dict, (size_t)(ch.dict_len * es), cudaMemcpyHostToDevice, ctx->stream));
  }
  WG_TRY(out.alloc(ctx, std::max<int64_t>(rows * oes, 16)));
  ChunkArgs a{};
  a.pages = (const PageD*)dpages.get();
  a.bytes = dbytes.as<uint8_t>();
  a.n_pages = ch.n_pages;
  a.es = (int32_t)es;
  a.widen = ch.type_id == WG_TYPE_DECIMAL;
  a.nullable = nullable;
  a.dict = ddict.get();
  a.dict_len = dict_enc ? ch.dict_len : 0;
  a.err = ctx->dev_error;
  a.rows = rows;
  DevBuf vbytes, wcnt, wpref, dense, scan_tmp;
  const int64_t nwords = (rows + 63) / 64;
  if (nullable && rows > 0) {
    WG_TRY(vbytes.alloc(ctx, rows));
    WG_TRY(out_valid.alloc(ctx, std::max<int64_t>(nwords, 1) * 8));
    WG_TRY(wcnt.alloc(ctx, (nwords + 1) * 8));
    WG_TRY(wpref.alloc(ctx, (nwords + 1) * 8));
    a.vbytes = vbytes.as<uint8_t>();
    def_levels_kernel<<<ch.n_pages, kPageThreads, 0, ctx->stream>>>(a);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    WG_CUDA_TRY(cudaMemsetAsync(wcnt.as<char>() + nwords * 8, 0, 8, ctx->stream));
    pack_valid_kernel<<<grid_for_rows(ctx, nwords, 256), 256, 0, ctx->stream>>>(
        vbytes.as<uint8_t>(), rows, out_valid.as<uint64_t>(), wcnt.as<unsigned long long>(), nwords);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, wcnt.as<unsigned long long>(), wpref.as<unsigned long long>(),
                                  (int)(nwords + 1), ctx->stream);
    WG_TRY(scan_tmp.alloc(ctx, std::max<int64_t>((int64_t)tb, 16)));
    cub::DeviceScan::ExclusiveSum(scan_tmp.get(), tb, wcnt.as<unsigned long long>(), wpref.as<unsigned long long>(),
                                  (int)(nwords + 1), ctx->stream);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    a.vwords = out_valid.as<uint64_t>();
    a.wprefix = wpref.as<unsigned long long>();
    int64_t nn = 0;
    WG_TRY(read_back_i64(ctx, (const int64_t*)(wpref.as<unsigned long long>() + nwords), &nn, 1));
    WG_TRY(dense.alloc(ctx, std::max<int64_t>(nn * oes, 16)));
    a.dense = dense.as<char>();
  } else {
    a.dense = out.as<char>();
  }
  if (rows > 0) {
    values_kernel<<<ch.n_pages, kPageThreads, 0, ctx->stream>>>(a);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
  }
  if (nullable && rows > 0) {
    scatter_kernel<<<grid_for_rows(ctx, rows, 256), 256, 0, ctx->stream>>>(a, out.as<char>(), (int)oes);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
  }
  *has_valid = nullable && rows > 0;
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // scratch and staging are released on return
  int32_t e = 0;
  WG_CUDA_TRY(cudaMemcpy(&e, ctx->dev_error, 4, cudaMemcpyDeviceToHost));
  if (e == WG_DERR_BAD_PAGE) {
    WG_CUDA_TRY(cudaMemset(ctx->dev_error, 0, 4));
    return fail(WG_E_INVALID, "malformed Parquet page (levels or indices end early, an index is past the "
                              "dictionary, or PLAIN data is shorter than its values)");
  }
  return check_device_error(ctx);
}

}  // namespace

extern "C" {

wg_status wg_batch_upload(wg_ctx* ctx, const wg_batch_desc* host, wg_batch** out) {
  if (!ctx || !host || !out) return fail(WG_E_INVALID, "NULL argument");
  *out = nullptr;
  WG_TRY(ensure_device(ctx));
  StagedBatch sb;
  WG_TRY(stage_batch(ctx, host, &sb));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  wg_batch* b = new wg_batch();
  b->ctx = ctx;
  b->data = std::move(sb.data);
  b->valid = std::move(sb.valid);
  b->sel = std::move(sb.sel);
  b->cols = sb.cols;
  b->len = host->len;
  b->has_sel = host->sel != nullptr;
  b->sel_len = host->sel_len;
  *out = b;
  return WG_OK;
}

wg_status wg_batch_decode(wg_ctx* ctx, const wg_column_chunk* chunks, int32_t n_chunks, wg_batch** out) {
  if (!ctx || !out || n_chunks < 1 || !chunks) return fail(WG_E_INVALID, "NULL argument");
  *out = nullptr;
  WG_TRY(ensure_device(ctx));
  int64_t rows = 0;
  for (int p = 0; p < chunks[0].n_pages; ++p) rows += chunks[0].pages[p].num_values;
  wg_batch* b = new wg_batch();
  b->ctx = ctx;
  b->len = rows;
  b->data.resize((size_t)n_chunks);
  b->valid.resize((size_t)n_chunks);
  for (int c = 0; c < n_chunks; ++c) {
    const wg_column_chunk& ch = chunks[c];
    if (ch.n_pages < 0 || (ch.n_pages > 0 && !ch.pages)) { delete b; return fail(WG_E_INVALID, "bad column chunk"); }
    bool hv = false;
    wg_status st = decode_chunk(ctx, ch, rows, b->data[(size_t)c], b->valid[(size_t)c], &hv);
    if (st != WG_OK) { delete b; return st; }
    wg_column col{};
    col.type_id = ch.type_id;
    col.scale = ch.scale;
    col.data = b->data[(size_t)c].get();
    col.valid_words = hv ? b->valid[(size_t)c].as<uint64_t>() : nullptr;
    col.len = rows;
    b->cols.push_back(col);
  }
  *out = b;
  return WG_OK;
}

wg_status wg_batch_device_desc(wg_batch* b, wg_batch_desc* out, wg_column* cols, int32_t max_cols) {
  if (!b || !out) return fail(WG_E_INVALID, "NULL argument");
  const int32_t n = (int32_t)b->cols.size();
  out->ncols = n;
  out->_pad = 0;
  out->len = b->len;
  out->sel = b->has_sel ? b->sel.as<uint32_t>() : nullptr;
  out->sel_len = b->has_sel ? b->sel_len : 0;
  out->cols = cols;
  if (!cols || max_cols < n) return fail(WG_E_INVALID, "cols has room for fewer columns than the batch holds");
  for (int32_t i = 0; i < n; ++i) cols[i] = b->cols[(size_t)i];
  return WG_OK;
}

wg_status wg_batch_destroy(wg_batch* b) {
  if (!b) return WG_OK;
  ensure_device(b->ctx);
  cudaStreamSynchronize(b->ctx->stream);
  delete b;
  return WG_OK;
}

}  // extern "C"
