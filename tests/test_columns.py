"""Host-side batch descriptors (no GPU): the STRING / BYTES column form that a
string GROUP BY key takes (batch.BytesColumn, internal/engine/batch/vector.go:92)."""
import ctypes as C

import numpy as np

import wadjet_b200 as wg
from wadjet_b200 import _abi as abi


def test_strings_column_layout_and_validity():
    col = wg.Column.strings(["ab", None, "", "héllo", b"\x00\x01"])
    offs, raw = col.data
    assert offs.dtype == np.uint32 and offs.tolist() == [0, 2, 2, 2, 8, 10]
    assert raw.tobytes() == b"ab" + "héllo".encode() + b"\x00\x01"
    assert col.valid.tolist() == [True, False, True, True, True]
    assert len(col) == 5
    assert wg.Column.strings(["x", "y"]).valid is None


def test_strings_descriptor_points_at_offsets_and_bytes():
    col = wg.Column.strings(["abc", "d"], wg.TYPE_BYTES)
    keep = []
    d = col._desc(keep)
    assert d.type_id == wg.TYPE_BYTES and d.len == 2 and not d.valid_words
    bd = abi.wg_bytes.from_address(d.data)
    offs = (C.c_uint32 * 3).from_address(bd.offsets)
    assert list(offs) == [0, 3, 4]
    assert C.string_at(bd.bytes, 4) == b"abcd"


def test_empty_strings_column():
    col = wg.Column.strings([])
    keep = []
    d = col._desc(keep)
    assert len(col) == 0 and d.len == 0
    bd = abi.wg_bytes.from_address(d.data)
    assert bd.offsets and bd.bytes  # valid pointers even with no bytes


def test_batch_with_a_string_column_and_selection():
    b = wg.Batch([wg.Column.strings(["a", "b", None]), wg.Column(wg.TYPE_INT64, np.arange(3, dtype=np.int64))],
                 sel=np.array([0, 2], np.uint32))
    d, keep = b.desc()
    assert d.ncols == 2 and d.len == 3 and d.sel_len == 2
    words = np.ctypeslib.as_array((C.c_uint64 * 1).from_address(d.cols[0].valid_words))
    assert int(words[0]) & 0b111 == 0b011
