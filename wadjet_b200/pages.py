"""Parquet data pages for the device decode entry point (wg_batch_decode).

`chunk()` builds the wg_column_chunk / wg_page descriptors over encoded page
bytes the caller already holds (a Parquet reader's pages after decompression).
`encode_plain`, `encode_dictionary` and `encode_levels` write flat-column data
pages the way a Parquet writer lays them out — PLAIN values of the non-NULL
rows; one bit-width byte and RLE / bit-packed hybrid indices for a dictionary
page; hybrid definition levels of bit width 1 — so tests and benchmarks can
hand synthetic tables over in their encoded form. The hybrid format is the
Parquet specification's (internal/storage/parquet/rle.go): a varint header,
even for a repeated value (count << 1, then ceil(bit_width / 8) value bytes),
odd for bit-packed groups of 8 values ((groups << 1) | 1, then groups *
bit_width bytes, values packed LSB first).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi as abi

ENC_PLAIN, ENC_PLAIN_DICTIONARY, ENC_RLE_DICTIONARY = abi.ENC_PLAIN, abi.ENC_PLAIN_DICTIONARY, abi.ENC_RLE_DICTIONARY


def _varint(v: int) -> bytes:
    out = bytearray()
    while v >= 0x80:
        out.append((v & 0x7F) | 0x80)
        v >>= 7
    out.append(v)
    return bytes(out)


def _bitpack(values: np.ndarray, bw: int) -> bytes:
    """values (a multiple of 8 of them) packed LSB first at bw bits each."""
    if bw == 0:
        return b""
    v = np.asarray(values, np.uint64)
    bits = ((v[:, None] >> np.arange(bw, dtype=np.uint64)) & np.uint64(1)).astype(np.uint8).reshape(-1)
    return np.packbits(bits, bitorder="little").tobytes()


def encode_hybrid(values: np.ndarray, bw: int, min_repeat: int = 8) -> bytes:
    """RLE / bit-packed hybrid of non-negative ints below 2^bw: runs of at least
    `min_repeat` equal values become repeated-value runs, the rest bit-packed
    groups of 8 (the last group padded with zeros)."""
    v = np.asarray(values, np.int64)
    n = len(v)
    out = bytearray()
    vb = (bw + 7) // 8
    i = 0
    pending: list[int] = []

    def flush_packed():
        nonlocal pending
        if not pending:
            return
        pad = (-len(pending)) % 8
        vals = np.array(pending + [0] * pad, np.uint64)
        out.extend(_varint(((len(vals) // 8) << 1) | 1))
        out.extend(_bitpack(vals, bw))
        pending = []

    while i < n:
        j = i
        while j < n and v[j] == v[i]:
            j += 1
        run = j - i
        # a repeated run may only start on a group boundary of the pending values
        if run >= min_repeat and len(pending) % 8 == 0:
            flush_packed()
            out.extend(_varint(run << 1))
            out.extend(int(v[i]).to_bytes(vb, "little") if vb else b"")
            i = j
        else:
            take = run if run < min_repeat else (8 - len(pending) % 8)
            pending.extend(int(x) for x in v[i:i + take])
            i += take
    flush_packed()
    return bytes(out)


def encode_levels(valid: np.ndarray) -> bytes:
    """Definition levels of an optional flat column (1 = value, 0 = NULL), bit width 1."""
    return encode_hybrid(np.asarray(valid, np.int64), 1)


def physical(values: np.ndarray, type_id: int) -> np.ndarray:
    """The PLAIN physical values of a column: DECIMAL (hi, lo) as its INT64 (the values must fit)."""
    if type_id == abi.TYPE_DECIMAL:
        hi, lo = values["hi"], values["lo"].view(np.int64)
        if not np.array_equal(hi, np.where(lo < 0, -1, 0)):
            raise ValueError("DECIMAL values wider than INT64 have no INT64 physical form")
        return lo
    return np.ascontiguousarray(values)


def encode_plain(values: np.ndarray, type_id: int, valid: Optional[np.ndarray] = None) -> bytes:
    v = physical(values, type_id)
    if valid is not None:
        v = v[np.asarray(valid, bool)]
    return np.ascontiguousarray(v).tobytes()


def encode_dictionary(values: np.ndarray, type_id: int, valid: Optional[np.ndarray] = None):
    """(dictionary values, page values section) of a dictionary-encoded page."""
    v = physical(values, type_id)
    if valid is not None:
        v = v[np.asarray(valid, bool)]
    dict_vals, idx = np.unique(v, return_inverse=True)
    bw = max(1, int(len(dict_vals) - 1).bit_length())
    return dict_vals, bytes([bw]) + encode_hybrid(idx.reshape(-1), bw)


@dataclass
class Page:
    num_values: int
    data: bytes
    encoding: int = ENC_PLAIN
    def_levels: Optional[bytes] = None


@dataclass
class Chunk:
    type_id: int
    pages: Sequence[Page]
    scale: int = 0
    dictionary: Optional[np.ndarray] = None
    _keep: list = field(default_factory=list)

    def to_c(self) -> "abi.wg_column_chunk":
        """The C descriptor; its pointers stay valid while this Chunk lives."""
        arr = (abi.wg_page * max(1, len(self.pages)))()
        keep = [arr]
        for i, p in enumerate(self.pages):
            d = np.frombuffer(p.data, np.uint8) if p.data else np.zeros(1, np.uint8)
            lv = np.frombuffer(p.def_levels, np.uint8) if p.def_levels else None
            keep += [d, lv]
            arr[i] = abi.wg_page(p.encoding, 0, p.num_values, lv.ctypes.data if lv is not None else None,
                                 len(p.def_levels) if p.def_levels else 0, d.ctypes.data, len(p.data))
        dptr, dlen = None, 0
        if self.dictionary is not None:
            dv = np.ascontiguousarray(self.dictionary)
            keep.append(dv)
            dptr, dlen = dv.ctypes.data, len(dv)
        self._keep = keep
        return abi.wg_column_chunk(self.type_id, self.scale, len(self.pages), 0, arr, dptr, dlen)


def chunk(values: np.ndarray, type_id: int, valid: Optional[np.ndarray] = None, page_rows: int = 1 << 17,
          dictionary: bool = False, scale: int = 0) -> Chunk:
    """A column as one chunk of data pages of `page_rows` rows (PLAIN or dictionary)."""
    n = len(values)
    pages = []
    dict_vals = None
    if dictionary:
        dict_vals, _ = np.unique(physical(values if valid is None else values[np.asarray(valid, bool)], type_id),
                                 return_inverse=True)
    for r0 in range(0, max(n, 1), page_rows):
        r1 = min(n, r0 + page_rows)
        v = values[r0:r1]
        ok = None if valid is None else np.asarray(valid[r0:r1], bool)
        levels = encode_levels(ok) if ok is not None else None
        if dictionary:
            phys = physical(v, type_id)
            if ok is not None:
                phys = phys[ok]
            idx = np.searchsorted(dict_vals, phys)
            bw = max(1, int(len(dict_vals) - 1).bit_length())
            data = bytes([bw]) + encode_hybrid(idx, bw)
            pages.append(Page(r1 - r0, data, ENC_RLE_DICTIONARY, levels))
        else:
            pages.append(Page(r1 - r0, encode_plain(v, type_id, ok), ENC_PLAIN, levels))
        if n == 0:
            break
    return Chunk(type_id, pages, scale, dict_vals)
