"""wadjet_b200 — Wadjet's filter → hash-join → hash-aggregate path on the B200.

A host-side mirror of the reference's operator contract
(internal/engine/exec/operators.go) over the C ABI of libwadjetgpu.so:

- ``KernelFilter``  — exec.KernelFilter (exec/filter.go:347): typed ``col OP const``
  that compacts the selection vector; ``None`` means "fully filtered".
- ``HashJoin``      — exec.HashJoin inner int-key join (exec/join.go:42): build,
  then bounded-output probe returning (probe_row, build_row) pairs.
- ``HashAggregate`` — exec.HashAggregate (exec/aggregate.go:98): consume batches,
  CloneSink / MergeSink, Finalize, then ``next()`` pages of 2048 rows.
- ``run_pipeline``  — Pipeline.Run (exec/pipeline.go:81) fused into one kernel.

Columns are numpy arrays (host) or torch CUDA tensors (device). DECIMAL values
use ``DEC_DTYPE`` = (hi int64, lo uint64), Go's batch.Int128 field order.
Every compute call runs on the GPU through the shared library; there is no CPU
fallback, and a missing library raises at import.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _abi as abi
from ._abi import (AGG_AVG, AGG_COUNT, AGG_MAX, AGG_MIN, AGG_SUM, CONST_FLOAT, CONST_INT, JOIN_ANTI, JOIN_INNER,
                   JOIN_LEFT, JOIN_SEMI, OP_EQ, OP_GE, OP_GT,
                   OP_LE, OP_LT, OP_NE, TYPE_BYTES, TYPE_DATE, TYPE_DECIMAL, TYPE_DURATION, TYPE_FLOAT32, TYPE_FLOAT64,
                   TYPE_INT32, TYPE_INT64, TYPE_IPV4, TYPE_MAC, TYPE_PORT, TYPE_PROTOCOL, TYPE_STRING,
                   TYPE_TIMESTAMP)

__all__ = [
    "Context", "Column", "Batch", "DeviceBatch", "KernelFilter", "HashJoin", "HashAggregate", "AggColumn", "Expr", "run_pipeline",
    "WadjetGPUError", "MemoryExceeded", "Cancelled", "DEC_DTYPE", "lib",
]

DEC_DTYPE = np.dtype([("hi", "<i8"), ("lo", "<u8")])
BATCH_SIZE = 2048  # batch.DefaultBatchSize (internal/engine/batch/batch.go:6)

class _Lib:
    """The loaded libwadjetgpu.so, opened on first use (so `python -m wadjet_b200.build`
    can run before the library exists). A missing library raises; nothing falls back."""

    def __getattr__(self, name):
        return getattr(abi.load(), name)


lib = _Lib()

_ELEM = {TYPE_INT32: 4, TYPE_PORT: 4, TYPE_PROTOCOL: 4, TYPE_DATE: 4, TYPE_FLOAT32: 4, TYPE_INT64: 8,
         TYPE_TIMESTAMP: 8, TYPE_IPV4: 8, TYPE_MAC: 8, TYPE_DURATION: 8, TYPE_FLOAT64: 8, TYPE_DECIMAL: 16}
_NP = {TYPE_INT32: np.int32, TYPE_PORT: np.int32, TYPE_PROTOCOL: np.int32, TYPE_DATE: np.int32,
       TYPE_FLOAT32: np.float32, TYPE_INT64: np.int64, TYPE_TIMESTAMP: np.int64, TYPE_IPV4: np.int64,
       TYPE_MAC: np.int64, TYPE_DURATION: np.int64, TYPE_FLOAT64: np.float64, TYPE_DECIMAL: DEC_DTYPE}


class WadjetGPUError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"wadjet-gpu status {status}: {msg}")
        self.status = status


class MemoryExceeded(WadjetGPUError):
    """memory.ErrMemoryExceeded (internal/engine/memory/tracker.go:15)."""


class Cancelled(WadjetGPUError):
    """A queued serving request was withdrawn (context.Canceled)."""


def _check(status: int) -> None:
    if status != abi.WG_OK:
        msg = (lib.wg_last_error() or b"").decode()
        if status == abi.WG_E_NOMEM:
            raise MemoryExceeded(status, msg)
        if status == abi.WG_E_CANCELLED:
            raise Cancelled(status, msg)
        raise WadjetGPUError(status, msg)


def pack_validity(valid: np.ndarray) -> np.ndarray:
    """bool per row (True = valid) → batch.Bitmap words (bit 1 = valid, LSB first)."""
    valid = np.asarray(valid, dtype=bool)
    b = np.packbits(valid, bitorder="little")
    pad = (-len(b)) % 8
    if pad:
        b = np.concatenate([b, np.zeros(pad, np.uint8)])
    return b.view(np.uint64).copy()


def unpack_validity(words: np.ndarray, n: int) -> np.ndarray:
    return np.unpackbits(np.asarray(words, np.uint64).view(np.uint8), bitorder="little")[:n].astype(bool)


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


@dataclass
class Column:
    """One batch.Vector: typed data plus optional validity (True = valid)."""
    type_id: int
    data: object                      # numpy array or torch tensor
    valid: Optional[object] = None    # numpy bool array / torch uint64 words on device
    scale: int = 0

    def __len__(self) -> int:
        if self.type_id in (TYPE_STRING, TYPE_BYTES):
            return int(self.data[0].shape[0]) - 1
        return int(self.data.shape[0])

    @classmethod
    def strings(cls, values: Sequence, type_id: int = TYPE_STRING) -> "Column":
        """A STRING / BYTES column (batch.BytesColumn) from str / bytes values, None = NULL:
        data is (offsets uint32[n + 1], bytes uint8)."""
        enc = [b"" if v is None else (v.encode() if isinstance(v, str) else bytes(v)) for v in values]
        offs = np.zeros(len(enc) + 1, np.uint32)
        if enc:
            offs[1:] = np.cumsum([len(b) for b in enc], dtype=np.uint64).astype(np.uint32)
        data = np.frombuffer(b"".join(enc), np.uint8).copy() if enc else np.zeros(0, np.uint8)
        valid = None
        if any(v is None for v in values):
            valid = np.array([v is not None for v in values], bool)
        return cls(type_id, (offs, data), valid)

    def _desc(self, keep: list) -> abi.wg_column:
        if self.type_id in (TYPE_STRING, TYPE_BYTES):
            # data = (offsets, bytes), numpy arrays or CUDA tensors; the column's
            # data pointer is a wg_bytes descriptor in host memory
            offs, raw = self.data
            if _is_torch(offs):
                desc = abi.wg_bytes(offs.data_ptr(), raw.data_ptr() if raw.numel() else offs.data_ptr())
                vptr = self.valid.data_ptr() if self.valid is not None else None
            else:
                o = np.ascontiguousarray(offs, dtype=np.uint32)
                b = np.ascontiguousarray(raw, dtype=np.uint8)
                if b.size == 0:
                    b = np.zeros(1, np.uint8)
                keep += [o, b]
                desc = abi.wg_bytes(o.ctypes.data, b.ctypes.data)
                vptr = None
                if self.valid is not None:
                    w = pack_validity(self.valid) if np.asarray(self.valid).dtype == bool else np.asarray(self.valid, np.uint64)
                    keep.append(w)
                    vptr = w.ctypes.data
            keep.append(desc)
            return abi.wg_column(self.type_id, 0, C.addressof(desc), vptr, len(self))
        if _is_torch(self.data):
            ptr = self.data.data_ptr()
            vptr = self.valid.data_ptr() if self.valid is not None else None
        else:
            arr = np.ascontiguousarray(self.data)
            keep.append(arr)
            ptr = arr.ctypes.data
            vptr = None
            if self.valid is not None:
                w = pack_validity(self.valid) if np.asarray(self.valid).dtype == bool else np.asarray(self.valid, np.uint64)
                keep.append(w)
                vptr = w.ctypes.data
        return abi.wg_column(self.type_id, self.scale, ptr, vptr, len(self))


class Batch:
    """batch.RecordBatch: columns plus an optional selection vector (ascending row ids)."""

    def __init__(self, cols: Sequence[Column], sel=None, length: Optional[int] = None):
        self.cols = list(cols)
        self.sel = sel
        self.len = length if length is not None else (len(self.cols[0]) if self.cols else 0)

    def desc(self) -> tuple[abi.wg_batch_desc, list]:
        keep: list = []
        arr = (abi.wg_column * max(1, len(self.cols)))(*[c._desc(keep) for c in self.cols])
        keep.append(arr)
        sel_ptr, sel_len = None, 0
        if self.sel is not None:
            if _is_torch(self.sel):
                sel_ptr, sel_len = self.sel.data_ptr(), int(self.sel.shape[0])
            else:
                s = np.ascontiguousarray(self.sel, dtype=np.uint32)
                keep.append(s)
                sel_ptr, sel_len = s.ctypes.data, len(s)
        d = abi.wg_batch_desc(len(self.cols), 0, arr, self.len, sel_ptr, sel_len)
        keep.append(d)
        return d, keep


class _DevColType:
    """Type facts of a device-batch column (what run_pipeline reads from a column)."""

    def __init__(self, type_id: int, scale: int, n: int):
        self.type_id, self.scale, self._n = type_id, scale, n

    def __len__(self) -> int:
        return self._n


class DeviceBatch:
    """A batch resident on the device (wg_batch): uploaded from a decoded host batch
    (`upload`) or decoded on the GPU from Parquet column chunks (`decode`). It stands
    in for a device-resident Batch in run_pipeline(..., device=True)."""

    def __init__(self, ctx: "Context", h, ncols: int):
        self.ctx, self.h = ctx, h
        cols = (abi.wg_column * max(1, ncols))()
        d = abi.wg_batch_desc()
        _check(lib.wg_batch_device_desc(h, C.byref(d), cols, ncols))
        self._d, self._arr = d, cols
        self.len = d.len
        self.sel = None
        self.cols = [_DevColType(cols[i].type_id, cols[i].scale, d.len) for i in range(ncols)]

    @classmethod
    def upload(cls, ctx: "Context", batch: Batch) -> "DeviceBatch":
        d, keep = batch.desc()
        h = C.c_void_p()
        _check(lib.wg_batch_upload(ctx.h, C.byref(d), C.byref(h)))
        return cls(ctx, h, len(batch.cols))

    @classmethod
    def decode(cls, ctx: "Context", chunks) -> "DeviceBatch":
        """chunks: wadjet_b200.pages.Chunk objects, one per column."""
        cs = [c.to_c() for c in chunks]
        arr = (abi.wg_column_chunk * len(cs))(*cs)
        h = C.c_void_p()
        _check(lib.wg_batch_decode(ctx.h, arr, len(cs), C.byref(h)))
        return cls(ctx, h, len(cs))

    def desc(self):
        return self._d, [self._arr]

    def column_pointer(self, i: int) -> tuple[int, int]:
        """(data, validity words) device addresses of column i (0 when it has no NULLs)."""
        c = self._arr[i]
        return int(c.data or 0), int(c.valid_words or 0)

    def close(self) -> None:
        if self.h:
            lib.wg_batch_destroy(self.h)
            self.h = None


class Context:
    """Device, stream and HBM ledger (memory.Tracker over device bytes)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, pinned_spill: int = 0):
        h = C.c_void_p()
        _check(lib.wg_ctx_create(device, hbm_budget, pinned_spill, C.byref(h)))
        self.h = h
        self.device = device

    def close(self) -> None:
        if self.h:
            lib.wg_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def synchronize(self) -> None:
        _check(lib.wg_ctx_synchronize(self.h))

    def ledger(self) -> dict:
        u, p, b = C.c_int64(), C.c_int64(), C.c_int64()
        _check(lib.wg_ledger_stats(self.h, C.byref(u), C.byref(p), C.byref(b)))
        return {"used": u.value, "peak": p.value, "budget": b.value}

    def reserve(self, n: int) -> None:
        _check(lib.wg_ledger_reserve(self.h, n))

    def release(self, n: int) -> None:
        _check(lib.wg_ledger_release(self.h, n))

    @property
    def stream(self) -> int:
        return lib.wg_ctx_stream(self.h) or 0

    @property
    def launches(self) -> int:
        return int(lib.wg_ctx_launch_count(self.h))


def _const(value) -> tuple[int, int, float]:
    if isinstance(value, (float, np.floating)):
        return CONST_FLOAT, 0, float(value)
    return CONST_INT, int(value), 0.0


class KernelFilter:
    """exec.KernelFilter: `batch.cols[col] OP value`; returns the compacted selection."""

    def __init__(self, ctx: Context, col: int, op: int, value):
        self.ctx = ctx
        kind, i, f = _const(value)
        h = C.c_void_p()
        _check(lib.wg_filter_create(ctx.h, col, op, kind, i, f, C.byref(h)))
        self.h = h

    def execute(self, batch: Batch) -> Optional[np.ndarray]:
        d, keep = batch.desc()
        n_items = len(batch.sel) if batch.sel is not None else batch.len
        out = np.empty(max(1, n_items), np.uint32)
        n = C.c_int64()
        _check(lib.wg_filter_execute(self.h, C.byref(d), out.ctypes.data, C.byref(n)))
        return None if n.value == 0 else out[: n.value].copy()

    def execute_device(self, batch: Batch, out_sel) -> int:
        d, keep = batch.desc()
        n = C.c_int64()
        _check(lib.wg_filter_execute_device(self.h, C.byref(d), out_sel.data_ptr(), C.byref(n)))
        return n.value

    def close(self) -> None:
        if self.h:
            lib.wg_filter_destroy(self.h)
            self.h = None


class HashJoin:
    """exec.HashJoin on one integer-class key + HashJoinProbe.

    join_type: JOIN_INNER, JOIN_LEFT (unmatched probe rows once, NULL build
    columns), JOIN_SEMI or JOIN_ANTI (probe rows only, no payload columns)."""

    def __init__(self, ctx: Context, build_key: int, probe_key: int, payload: Sequence[int] = (),
                 build_row_hint: int = 0, join_type: int = abi.JOIN_INNER):
        self.ctx = ctx
        self.payload = list(payload)
        self.payload_types: list[int] = []
        self.join_type = join_type
        pay = (C.c_int32 * max(1, len(payload)))(*payload)
        h = C.c_void_p()
        _check(lib.wg_join_create(ctx.h, join_type, build_key, probe_key, len(payload), pay, build_row_hint,
                                  C.byref(h)))
        self.h = h

    def build(self, batches: Iterable[Batch], device: bool = False) -> None:
        for b in batches:
            if not self.payload_types:
                self.payload_types = [b.cols[p].type_id for p in self.payload]
            d, keep = b.desc()
            fn = lib.wg_join_build_append_device if device else lib.wg_join_build_append
            _check(fn(self.h, C.byref(d)))
        _check(lib.wg_join_build_finish(self.h))

    def reset(self) -> None:
        """Forget the build side (device buffers are kept for the next build)."""
        _check(lib.wg_join_reset(self.h))

    def stats(self) -> tuple[int, int]:
        r, k = C.c_int64(), C.c_int64()
        _check(lib.wg_join_build_stats(self.h, C.byref(r), C.byref(k)))
        return r.value, k.value

    def probe(self, batch: Batch, cap: int = 16 * BATCH_SIZE):
        """Yield (probe_rows uint32, build_rows int64) chunks of at most `cap` pairs."""
        d, keep = batch.desc()
        cursor = C.c_int64(0)
        while True:
            pr = np.empty(max(1, cap), np.uint32)
            br = np.empty(max(1, cap), np.int64)
            n = C.c_int64()
            _check(lib.wg_join_probe(self.h, C.byref(d), pr.ctypes.data, br.ctypes.data, cap, C.byref(cursor),
                                     C.byref(n)))
            if n.value > 0:
                yield pr[: n.value].copy(), br[: n.value].copy()
            if n.value < cap:
                return

    def bloom_filter(self, batch: Batch) -> np.ndarray:
        """BloomFilterOp.Execute: the rows (or selection entries) whose probe key the build side's
        bloom filter may contain, ascending."""
        d, keep = batch.desc()
        n_items = len(batch.sel) if batch.sel is not None else batch.len
        out = np.empty(max(1, n_items), np.uint32)
        n = C.c_int64()
        _check(lib.wg_join_bloom_filter(self.h, C.byref(d), out.ctypes.data, C.byref(n)))
        return out[: n.value].copy()

    def gather(self, payload_idx: int, build_rows: np.ndarray, dtype) -> tuple[np.ndarray, np.ndarray]:
        rows = np.ascontiguousarray(build_rows, np.int64)
        out = np.empty(max(1, len(rows)), dtype)
        valid = np.empty(max(1, len(rows)), np.uint8)
        _check(lib.wg_join_gather(self.h, payload_idx, rows.ctypes.data, len(rows), out.ctypes.data,
                                  valid.ctypes.data))
        return out[: len(rows)], valid[: len(rows)].astype(bool)

    def close(self) -> None:
        if self.h:
            lib.wg_join_destroy(self.h)
            self.h = None


@dataclass
class AggColumn:
    """exec.AggColumn: func, input column (-1 = COUNT(*)), declared output type (0 = default)."""
    func: int
    input_col: int = -1
    out_type: int = 0


class HashAggregate:
    """exec.HashAggregate over the device hash table."""

    def __init__(self, ctx: Context, group_by: Sequence[int], aggs: Sequence[AggColumn], ndv_hint: int = 0,
                 _handle=None):
        self.ctx = ctx
        self.group_by = list(group_by)
        self.aggs = list(aggs)
        self.ndv_hint = ndv_hint
        self._key_types: Optional[list[int]] = None
        if _handle is not None:
            self.h = _handle
            return
        keys = (C.c_int32 * max(1, len(group_by)))(*group_by)
        specs = (abi.wg_agg_spec * max(1, len(aggs)))(*[abi.wg_agg_spec(a.func, a.input_col, a.out_type, 0)
                                                        for a in aggs])
        h = C.c_void_p()
        _check(lib.wg_agg_create(ctx.h, len(group_by), keys, len(aggs), specs, ndv_hint, C.byref(h)))
        self.h = h
        self._out_pos = 0
        self._n_groups = None

    def consume(self, batch: Batch, device: bool = False) -> None:
        if self._key_types is None:
            self._key_types = [batch.cols[k].type_id for k in self.group_by]
            self._in_types = [batch.cols[a.input_col].type_id if a.input_col >= 0 else None for a in self.aggs]
        d, keep = batch.desc()
        _check((lib.wg_agg_consume_device if device else lib.wg_agg_consume)(self.h, C.byref(d)))

    def clone_sink(self) -> "HashAggregate":
        h = C.c_void_p()
        _check(lib.wg_agg_clone(self.h, C.byref(h)))
        c = HashAggregate(self.ctx, self.group_by, self.aggs, self.ndv_hint, _handle=h)
        c._out_pos, c._n_groups = 0, None
        return c

    def merge_sink(self, other: "HashAggregate") -> None:
        _check(lib.wg_agg_merge(self.h, other.h))
        if self._key_types is None and other._key_types is not None:
            self._key_types, self._in_types = other._key_types, other._in_types

    def finalize(self) -> int:
        n = C.c_int64()
        _check(lib.wg_agg_finalize(self.h, C.byref(n)))
        self._n_groups = n.value
        self._out_pos = 0
        return n.value

    def reset(self) -> None:
        _check(lib.wg_agg_reset(self.h))
        self._n_groups = None
        self._out_pos = 0

    def state_layout(self) -> "abi.wg_state_layout":
        """The row layout of this aggregate's partial state (wg_agg_state_layout)."""
        lay = abi.wg_state_layout()
        _check(lib.wg_agg_state_layout(self.h, C.byref(lay)))
        return lay

    def partition_state(self, n_parts: int):
        """After finalize: every group's state row on the device, grouped by owner rank
        (partitionFor over the key's route hash). Returns (rows, part_rows): rows is a
        uint64 CUDA tensor of shape (groups, 1 + slot_words), part_rows the rows per owner."""
        import torch
        n = self.finalize()
        lay = self.state_layout() if n else None
        width = 1 + (lay.slot_words if lay is not None else 0)
        rows = torch.empty((max(n, 1), max(width, 1)), dtype=torch.int64, device=f"cuda:{self.ctx.device}")
        counts = (C.c_int64 * n_parts)()
        _check(lib.wg_agg_partition_state(self.h, n_parts, rows.data_ptr(), n, counts))
        return rows[:n], [int(c) for c in counts]

    def merge_state(self, layout: "abi.wg_state_layout", rows) -> None:
        """MergeSink of state rows (a CUDA tensor of shape (n, 1 + slot_words)) laid out as `layout`."""
        n = int(rows.shape[0]) if rows is not None else 0
        ptr = rows.data_ptr() if n else None
        _check(lib.wg_agg_merge_state(self.h, C.byref(layout), ptr, n))

    @property
    def kernel_shape(self) -> int:
        """Compiled query shape of the last fused launch (0 generic, -1 none yet); a diagnostic only."""
        return int(lib.wg_agg_kernel_shape(self.h))

    def export(self) -> dict:
        """Raw accumulator state of every group (keys widened to int64)."""
        n = self._n_groups if self._n_groups is not None else self.finalize()
        nk, na = len(self.group_by), len(self.aggs)
        r = {"keys": np.zeros((nk, n), np.int64), "key_valid": np.zeros((nk, n), np.uint8),
             "count": np.zeros((na, n), np.int64), "i64": np.zeros((na, n), np.int64),
             "f64": np.zeros((na, n), np.float64), "dec": np.zeros((na, n), DEC_DTYPE),
             "has": np.zeros((na, n), np.uint8)}
        if n == 0:
            return r
        e = abi.wg_group_export(*[r[k].ctypes.data if r[k].size else None
                                  for k in ("keys", "key_valid", "count", "i64", "f64", "dec", "has")])
        _check(lib.wg_agg_export(self.h, C.byref(e)))
        return r

    @property
    def string_keyed(self) -> bool:
        """Grouped by one STRING / BYTES column: the table keys its groups by dense ids."""
        return bool(self._key_types) and self._key_types[0] in (TYPE_STRING, TYPE_BYTES)

    def key_strings(self, ids) -> list[bytes]:
        """The strings of dictionary ids (wg_agg_key_strings), as bytes."""
        ids = np.ascontiguousarray(ids, dtype=np.int64)
        n = len(ids)
        offs = np.zeros(n + 1, np.uint32)
        need = C.c_int64()
        cap = 1 << 16
        while True:
            buf = np.zeros(max(cap, 1), np.uint8)
            _check(lib.wg_agg_key_strings(self.h, ids.ctypes.data_as(C.POINTER(C.c_int64)), n, offs.ctypes.data,
                                          buf.ctypes.data, cap, C.byref(need)))
            if need.value <= cap:
                break
            cap = need.value
        raw = buf.tobytes()
        return [raw[offs[i]:offs[i + 1]] for i in range(n)]

    def output_types(self) -> list[int]:
        key_types = self._key_types or [TYPE_INT64] * len(self.group_by)
        key_types = [TYPE_INT32 if t in (TYPE_STRING, TYPE_BYTES) else t for t in key_types]
        outs = []
        for i, a in enumerate(self.aggs):
            if a.out_type:
                outs.append(a.out_type)
            elif a.func == AGG_COUNT:
                outs.append(TYPE_INT64)
            elif a.func in (AGG_SUM, AGG_AVG):
                outs.append(TYPE_FLOAT64)
            else:
                t = self._in_types[i] if self._key_types is not None else None
                outs.append(TYPE_FLOAT64 if t in (TYPE_FLOAT32, TYPE_FLOAT64, TYPE_DECIMAL, None) else TYPE_INT64)
        return [t if _ELEM.get(t) == 4 else (TYPE_INT64 if t != TYPE_FLOAT64 else t) for t in key_types] + outs

    def next(self, max_rows: int = BATCH_SIZE) -> Optional[list[tuple[np.ndarray, np.ndarray]]]:
        """HashAggregate.Next: the next page of finalized rows as (values, valid) per column, or None."""
        if self._n_groups is None:
            self.finalize()
        if self._out_pos >= self._n_groups:
            return None
        m = min(max_rows, self._n_groups - self._out_pos)
        types = self.output_types()
        bufs, words = [], []
        cols = (abi.wg_column * len(types))()
        for i, t in enumerate(types):
            b = np.zeros(m, np.int32 if _ELEM.get(t) == 4 else (np.float64 if t == TYPE_FLOAT64 else np.int64))
            w = np.zeros((m + 63) // 64, np.uint64)
            bufs.append(b)
            words.append(w)
            cols[i] = abi.wg_column(t, 0, b.ctypes.data, w.ctypes.data, m)
        n = C.c_int64()
        _check(lib.wg_agg_emit(self.h, self._out_pos, m, cols, C.byref(n)))
        self._out_pos += n.value
        out = [(b[: n.value], unpack_validity(w, n.value)) for b, w in zip(bufs, words)]
        if self.string_keyed:  # ids back to their strings (None for the NULL key)
            ids, ok = out[0]
            strs = self.key_strings(ids[ok])
            col = np.empty(n.value, object)
            col[ok] = strs
            if self._key_types[0] == TYPE_STRING:
                col[ok] = [x.decode() for x in strs]
            out[0] = (col, ok)
        return out

    def collect(self) -> list[tuple[np.ndarray, np.ndarray]]:
        """Every finalized row (all pages of next() concatenated)."""
        pages = []
        while True:
            p = self.next(1 << 20)
            if p is None:
                break
            pages.append(p)
        if not pages:
            types = self.output_types()
            return [(np.zeros(0, np.int32 if _ELEM.get(t) == 4 else (np.float64 if t == TYPE_FLOAT64 else np.int64)),
                     np.zeros(0, bool)) for t in types]
        return [(np.concatenate([p[i][0] for p in pages]), np.concatenate([p[i][1] for p in pages]))
                for i in range(len(pages[0]))]

    def close(self) -> None:
        if self.h:
            lib.wg_agg_destroy(self.h)
            self.h = None


class Expr:
    """Postfix projection program: Expr.float_([Expr.col(3), Expr.const_f(1.0), Expr.col(4), "-", "*"])."""

    _OPS = {"+": abi.EXPR_ADD, "-": abi.EXPR_SUB, "*": abi.EXPR_MUL, "/": abi.EXPR_DIV, ">>": abi.EXPR_SHR,
            "&": abi.EXPR_AND}

    def __init__(self, result_type: int, program: Sequence):
        self.result_type = result_type
        self.program = list(program)

    @staticmethod
    def col(i: int):
        return ("col", i)

    @staticmethod
    def const_i(v: int):
        return ("ci", v)

    @staticmethod
    def const_f(v: float):
        return ("cf", v)

    def to_c(self) -> abi.wg_expr:
        e = abi.wg_expr()
        e.result_type = self.result_type
        e.n_ops = len(self.program)
        for k, op in enumerate(self.program):
            if isinstance(op, str):
                e.ops[k] = abi.wg_expr_op(self._OPS[op], 0, 0, 0.0)
            elif op[0] == "col":
                e.ops[k] = abi.wg_expr_op(abi.EXPR_COL, op[1], 0, 0.0)
            elif op[0] == "ci":
                e.ops[k] = abi.wg_expr_op(abi.EXPR_CONST_I, 0, int(op[1]), 0.0)
            else:
                e.ops[k] = abi.wg_expr_op(abi.EXPR_CONST_F, 0, 0, float(op[1]))
        return e


def _export_arrays(nk: int, na: int, n: int) -> dict:
    return {"keys": np.zeros((nk, n), np.int64), "key_valid": np.zeros((nk, n), np.uint8),
            "count": np.zeros((na, n), np.int64), "i64": np.zeros((na, n), np.int64),
            "f64": np.zeros((na, n), np.float64), "dec": np.zeros((na, n), DEC_DTYPE),
            "has": np.zeros((na, n), np.uint8)}


@dataclass
class TuneParams:
    """Launch shape / table sizing of the batched mode (wg_tune_params); 0 = default."""
    tile_rows: int = 0
    block: int = 0
    ctas_per_sm: int = 0
    smem_max_groups: int = 0
    max_load: float = 0.0


class BatchedQueries:
    """Many independent filter + probe + GROUP BY queries run by one persistent launch
    replayed from a CUDA graph. queries: list of dicts with keys
    batch (device Batch), group_by, aggs (AggColumn), filters [(col, op, value)], ndv_hint,
    and optionally join (a built HashJoin) and exprs (Expr) over the virtual schema."""

    def __init__(self, ctx: Context, queries: Sequence[dict], params: Optional[TuneParams] = None):
        self.ctx = ctx
        self._keep: list = []
        self.shapes = []
        arr = (abi.wg_batched_query * len(queries))()
        for i, q in enumerate(queries):
            d, keep = q["batch"].desc()
            self._keep += [d, keep]
            f = (abi.wg_predicate * max(1, len(q.get("filters", ()))))(*[predicate(*x) for x in q.get("filters", ())])
            keys = (C.c_int32 * max(1, len(q["group_by"])))(*q["group_by"])
            specs = (abi.wg_agg_spec * max(1, len(q["aggs"])))(*[abi.wg_agg_spec(a.func, a.input_col, a.out_type, 0)
                                                                 for a in q["aggs"]])
            exprs = list(q.get("exprs", ()))
            ex = (abi.wg_expr * max(1, len(exprs)))(*[e.to_c() for e in exprs])
            join = q.get("join")
            self._keep += [f, keys, specs, ex, join]
            arr[i] = abi.wg_batched_query(C.pointer(d), len(q.get("filters", ())), len(q["aggs"]), f, keys,
                                          len(q["group_by"]), len(exprs), specs, int(q.get("ndv_hint", 0)),
                                          join.h if join is not None else None, ex)
            self.shapes.append((len(q["group_by"]), len(q["aggs"])))
        self._keep.append(arr)
        tp = params or TuneParams()
        ctp = abi.wg_tune_params(tp.tile_rows, tp.block, tp.ctas_per_sm, tp.smem_max_groups, tp.max_load)
        h = C.c_void_p()
        _check(lib.wg_batched_create(ctx.h, len(queries), arr, C.byref(ctp), C.byref(h)))
        self.h = h
        self.n = len(queries)

    def run(self) -> np.ndarray:
        out = np.zeros(self.n, np.int64)
        _check(lib.wg_batched_run(self.h, out.ctypes.data_as(C.POINTER(C.c_int64))))
        return out

    def export(self, q: int, n_groups: int) -> dict:
        nk, na = self.shapes[q]
        r = _export_arrays(nk, na, n_groups)
        if n_groups:
            e = abi.wg_group_export(*[r[k].ctypes.data if r[k].size else None
                                      for k in ("keys", "key_valid", "count", "i64", "f64", "dec", "has")])
            _check(lib.wg_batched_export(self.h, q, C.byref(e)))
        return r

    def close(self) -> None:
        if self.h:
            lib.wg_batched_destroy(self.h)
            self.h = None


class Server:
    """Continuous-batching request loop over device-resident tables (wg_server_*).

    submit(batch, group_by, aggs, filters=(), join=None, exprs=(), ndv_hint=0) → ticket;
    wait(ticket) → (n_groups, latency_s); export(ticket, n_groups) → raw group state;
    release(ticket) frees the result (its aggregate returns to the slot's pool)."""

    def __init__(self, ctx: Context, slots: int):
        self.ctx = ctx
        h = C.c_void_p()
        _check(lib.wg_server_create(ctx.h, slots, C.byref(h)))
        self.h = h
        self._shapes: dict[int, tuple[int, int]] = {}

    def submit(self, batch: Batch, group_by: Sequence[int], aggs: Sequence[AggColumn], filters: Sequence = (),
               join: Optional["HashJoin"] = None, exprs: Sequence[Expr] = (), ndv_hint: int = 0,
               est_bytes: int = 0) -> int:
        d, keep = batch.desc()
        preds = (abi.wg_predicate * max(1, len(filters)))(*[predicate(*f) for f in filters])
        ex = (abi.wg_expr * max(1, len(exprs)))(*[e.to_c() for e in exprs])
        p = abi.wg_pipeline_desc(C.pointer(d), len(filters), len(exprs), preds, join.h if join else None, ex, None)
        keys = (C.c_int32 * max(1, len(group_by)))(*group_by)
        specs = (abi.wg_agg_spec * max(1, len(aggs)))(*[abi.wg_agg_spec(a.func, a.input_col, a.out_type, 0)
                                                        for a in aggs])
        r = abi.wg_serve_request(C.pointer(p), keys, specs, len(group_by), len(aggs), ndv_hint, est_bytes)
        t = C.c_int64()
        _check(lib.wg_server_submit(self.h, C.byref(r), C.byref(t)))
        self._shapes[t.value] = (len(group_by), len(aggs))
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0) -> tuple[int, float]:
        n, lat = C.c_int64(), C.c_double()
        _check(lib.wg_server_wait(self.h, ticket, timeout, C.byref(n), C.byref(lat)))
        return n.value, lat.value

    def export(self, ticket: int, n_groups: int) -> dict:
        nk, na = self._shapes[ticket]
        r = _export_arrays(nk, na, n_groups)
        if n_groups:
            e = abi.wg_group_export(*[r[k].ctypes.data if r[k].size else None
                                      for k in ("keys", "key_valid", "count", "i64", "f64", "dec", "has")])
            _check(lib.wg_server_export(self.h, ticket, C.byref(e)))
        return r

    def release(self, ticket: int) -> None:
        _check(lib.wg_server_release(self.h, ticket))
        self._shapes.pop(ticket, None)

    def cancel(self, ticket: int) -> None:
        """Withdraw a request that is still queued; its wait() then raises Cancelled."""
        _check(lib.wg_server_cancel(self.h, ticket))

    def stats(self) -> dict:
        s = abi.wg_serve_stats()
        _check(lib.wg_server_stats(self.h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in abi.wg_serve_stats._fields_}

    def reset_stats(self) -> None:
        _check(lib.wg_server_reset_stats(self.h))

    def close(self) -> None:
        if self.h:
            lib.wg_server_destroy(self.h)
            self.h = None


def predicate(col: int, op: int, value) -> abi.wg_predicate:
    kind, i, f = _const(value)
    return abi.wg_predicate(col, op, kind, 0, i, f)


def run_pipeline(ctx: Context, batch: Batch, agg: HashAggregate, filters: Sequence = (),
                 join: Optional[HashJoin] = None, exprs: Sequence[Expr] = (), device: bool = False) -> None:
    """Pipeline.Run: KernelFilter* → HashJoinProbe → Project → HashAggregate in one kernel per window.

    `filters` are (col, op, value) triples on input columns. The aggregate sees
    the virtual schema [input columns, join payload columns, expressions].
    """
    d, keep = batch.desc()
    preds = (abi.wg_predicate * max(1, len(filters)))(*[predicate(*f) for f in filters])
    ex = (abi.wg_expr * max(1, len(exprs)))(*[e.to_c() for e in exprs])
    if agg._key_types is None:
        pay_types = getattr(join, "payload_types", [])
        vtypes = [c.type_id for c in batch.cols] + list(pay_types) + [e.result_type for e in exprs]
        agg._key_types = [vtypes[k] for k in agg.group_by]
        agg._in_types = [vtypes[a.input_col] if a.input_col >= 0 else None for a in agg.aggs]
    p = abi.wg_pipeline_desc(C.pointer(d), len(filters), len(exprs), preds, join.h if join else None, ex, agg.h)
    _check((lib.wg_pipeline_run_device if device else lib.wg_pipeline_run)(ctx.h, C.byref(p)))
