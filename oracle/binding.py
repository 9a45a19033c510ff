"""TEST INFRASTRUCTURE ONLY — ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

The oracle restates Wadjet's CPU semantics for the filter → hash-join →
hash-aggregate path (see oracle/oracle.h for the reference file:line each
function follows). Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "liboracle.so")

DEC_DTYPE = np.dtype([("hi", "<i8"), ("lo", "<u8")])


class Column(C.Structure):
    _fields_ = [("type_id", C.c_int32), ("scale", C.c_int32), ("data", C.c_void_p),
                ("valid_words", C.c_void_p), ("len", C.c_int64)]


class BatchDesc(C.Structure):
    _fields_ = [("ncols", C.c_int32), ("_pad", C.c_int32), ("cols", C.POINTER(Column)),
                ("len", C.c_int64), ("sel", C.c_void_p), ("sel_len", C.c_int64)]


class AggSpec(C.Structure):
    _fields_ = [("func", C.c_int32), ("input_col", C.c_int32), ("out_type", C.c_int32), ("_pad", C.c_int32)]


class Predicate(C.Structure):
    _fields_ = [("col", C.c_int32), ("op", C.c_int32), ("const_kind", C.c_int32), ("_pad", C.c_int32),
                ("const_i64", C.c_int64), ("const_f64", C.c_double)]


class ExprOp(C.Structure):
    _fields_ = [("opcode", C.c_int32), ("arg", C.c_int32), ("imm_i64", C.c_int64), ("imm_f64", C.c_double)]


class Expr(C.Structure):
    _fields_ = [("result_type", C.c_int32), ("n_ops", C.c_int32), ("ops", ExprOp * 12)]


class GroupExport(C.Structure):
    _fields_ = [("keys", C.c_void_p), ("key_valid", C.c_void_p), ("count", C.c_void_p), ("i64", C.c_void_p),
                ("f64", C.c_void_p), ("dec", C.c_void_p), ("has", C.c_void_p)]


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        sig = {
            "or_last_error": (C.c_char_p, []),
            "or_filter": (I64, [C.POINTER(Column), I64, P, I64, C.POINTER(Predicate), P]),
            "or_join_new": (P, [I64]),
            "or_join_bloom_filter": (I64, [P, C.POINTER(Column), I64, P, I64, P, P]),
            "or_join_append": (C.c_int, [P, C.POINTER(Column), I64]),
            "or_join_rows": (I64, [P]),
            "or_join_distinct": (I64, [P]),
            "or_join_probe": (I64, [P, C.POINTER(Column), I64, P, I64, P, P, I64]),
            "or_join_free": (None, [P]),
            "or_join_set_type": (None, [P, I32]),
            "or_agg_new": (P, [I32, P, I32, P]),
            "or_agg_consume": (C.c_int, [P, C.POINTER(BatchDesc)]),
            "or_agg_groups": (I64, [P]),
            "or_agg_export": (C.c_int, [P, C.POINTER(GroupExport)]),
            "or_agg_emit": (C.c_int, [P, C.POINTER(Column)]),
            "or_agg_merge": (C.c_int, [P, P]),
            "or_agg_clone": (P, [P]),
            "or_agg_free": (None, [P]),
            "or_pipeline_run": (C.c_int, [C.POINTER(BatchDesc), I32, P, P, I32, C.POINTER(BatchDesc), I32, P, I32,
                                          P, P, I32]),
            "or_gen_starjoin_fact": (None, [C.c_uint64, I64, I64, P, P, P, P, I32]),
            "or_gen_starjoin_dim": (None, [C.c_uint64, I64, P, P]),
            "or_gen_groupby": (None, [C.c_uint64, I64, I64, I64, P, P, P, P, I32]),
            "or_gen_highcard": (None, [C.c_uint64, I64, I64, P, P, P, P, I32]),
            "or_i128_to_f64": (C.c_double, [I64, C.c_uint64, I32]),
            "or_rle_decode": (I64, [P, I64, I32, I64, P]),
            "or_page_decode": (C.c_int, [P, P, P]),
            "or_strindex_new": (P, []),
            "or_strindex_map": (I64, [P, P, P, P, I64, P, I64, P]),
            "or_strindex_get": (I64, [P, I64, P, I64]),
            "or_strindex_free": (None, [P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _err() -> str:
    return (lib().or_last_error() or b"").decode()


def _ptr(a):
    return None if a is None else a.ctypes.data


def pack_validity(valid) -> np.ndarray:
    b = np.packbits(np.asarray(valid, bool), bitorder="little")
    pad = (-len(b)) % 8
    if pad:
        b = np.concatenate([b, np.zeros(pad, np.uint8)])
    return b.view(np.uint64).copy()


class HostBatch:
    """A host batch of numpy columns: list of (type_id, array, valid_bool_or_None, scale)."""

    def __init__(self, cols, sel=None, length=None):
        self.keep = []
        arr = (Column * max(1, len(cols)))()
        n = length
        for i, (t, data, valid, scale) in enumerate(cols):
            data = np.ascontiguousarray(data)
            self.keep.append(data)
            w = None
            if valid is not None:
                w = pack_validity(valid)
                self.keep.append(w)
            arr[i] = Column(t, scale, data.ctypes.data, _ptr(w), len(data))
            n = len(data) if n is None else n
        self.arr = arr
        s = None
        if sel is not None:
            s = np.ascontiguousarray(sel, np.uint32)
            self.keep.append(s)
        self.desc = BatchDesc(len(cols), 0, arr, n or 0, _ptr(s), 0 if s is None else len(s))


def filter_(t, data, valid, op, value, sel=None) -> np.ndarray:
    hb = HostBatch([(t, data, valid, 0)])  # keeps the column and its packed validity alive for the call
    kind, i, f = (1, 0, float(value)) if isinstance(value, float) else (0, int(value), 0.0)
    p = Predicate(0, op, kind, 0, i, f)
    s = None if sel is None else np.ascontiguousarray(sel, np.uint32)
    out = np.empty(max(1, len(data) if s is None else len(s)), np.uint32)
    n = lib().or_filter(C.byref(hb.arr[0]), len(data), _ptr(s), 0 if s is None else len(s), C.byref(p),
                        out.ctypes.data)
    if n < 0:
        raise RuntimeError(_err())
    return out[:n].copy()


class Join:
    def __init__(self, hint=64, join_type=0):
        self.h = lib().or_join_new(hint)
        self.rows = 0
        if join_type:
            lib().or_join_set_type(self.h, join_type)

    def append(self, t, keys, valid=None):
        b = HostBatch([(t, keys, valid, 0)])
        if lib().or_join_append(self.h, C.byref(b.arr[0]), self.rows) != 0:
            raise RuntimeError(_err())
        self.rows += len(keys)

    def probe(self, t, keys, valid=None, sel=None):
        b = HostBatch([(t, keys, valid, 0)], sel=sel)
        s = b.keep[-1] if sel is not None else None
        sp, sl = (_ptr(s), len(s)) if s is not None else (None, 0)
        total = lib().or_join_probe(self.h, C.byref(b.arr[0]), len(keys), sp, sl, None, None, 0)
        pr = np.empty(max(1, total), np.uint32)
        br = np.empty(max(1, total), np.int64)
        lib().or_join_probe(self.h, C.byref(b.arr[0]), len(keys), sp, sl, pr.ctypes.data, br.ctypes.data, total)
        return pr[:total], br[:total]

    def distinct(self):
        return lib().or_join_distinct(self.h)

    def bloom_filter(self, t, keys, valid=None, sel=None):
        """BloomFilterOp.Execute over one int key column: (selected rows, bloom words)."""
        b = HostBatch([(t, keys, valid, 0)], sel=sel)
        s = b.keep[-1] if sel is not None else None
        sp, sl = (_ptr(s), len(s)) if s is not None else (None, 0)
        out = np.empty(max(1, len(keys) if s is None else len(s)), np.uint32)
        nw = C.c_int64()
        n = lib().or_join_bloom_filter(self.h, C.byref(b.arr[0]), len(keys), sp, sl, out.ctypes.data, C.byref(nw))
        if n < 0:
            raise RuntimeError(_err())
        return out[:n].copy(), nw.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_join_free(self.h)
            self.h = None


class Agg:
    def __init__(self, group_by, aggs):
        """aggs: list of (func, input_col, out_type)."""
        self.nk, self.na = len(group_by), len(aggs)
        keys = (C.c_int32 * max(1, self.nk))(*group_by)
        specs = (AggSpec * max(1, self.na))(*[AggSpec(f, c, o, 0) for f, c, o in aggs])
        self.h = lib().or_agg_new(self.nk, keys, self.na, specs)

    def consume(self, batch: HostBatch):
        if lib().or_agg_consume(self.h, C.byref(batch.desc)) != 0:
            raise RuntimeError(_err())

    def merge(self, other: "Agg"):
        if lib().or_agg_merge(self.h, other.h) != 0:
            raise RuntimeError(_err())

    def groups(self) -> int:
        return lib().or_agg_groups(self.h)

    def export(self) -> dict:
        n = self.groups()
        r = {"keys": np.zeros((self.nk, n), np.int64), "key_valid": np.zeros((self.nk, n), np.uint8),
             "count": np.zeros((self.na, n), np.int64), "i64": np.zeros((self.na, n), np.int64),
             "f64": np.zeros((self.na, n), np.float64), "dec": np.zeros((self.na, n), DEC_DTYPE),
             "has": np.zeros((self.na, n), np.uint8)}
        if n:
            e = GroupExport(*[r[k].ctypes.data if r[k].size else None
                              for k in ("keys", "key_valid", "count", "i64", "f64", "dec", "has")])
            lib().or_agg_export(self.h, C.byref(e))
        return r

    def emit(self, out_types) -> list:
        """Finalized columns [(values, valid)] for out_types (numpy dtypes per output column)."""
        n = self.groups()
        cols = (Column * len(out_types))()
        bufs = []
        for i, dt in enumerate(out_types):
            b = np.zeros(max(1, n), dt)
            w = np.zeros(max(1, (n + 63) // 64), np.uint64)
            bufs.append((b, w))
            cols[i] = Column(0, 0, b.ctypes.data, w.ctypes.data, n)
        lib().or_agg_emit(self.h, cols)
        return [(b[:n], np.unpackbits(w.view(np.uint8), bitorder="little")[:n].astype(bool)) for b, w in bufs]

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_agg_free(self.h)
            self.h = None


def pipeline(batch: HostBatch, agg: Agg, filters=(), join: Join = None, probe_key=-1, build: HostBatch = None,
             payload=(), exprs=(), threads=1):
    """filters: (col, op, value); exprs: Expr structures (same layout as wg_expr)."""
    preds = (Predicate * max(1, len(filters)))()
    for i, (c, op, v) in enumerate(filters):
        kind, iv, fv = (1, 0, float(v)) if isinstance(v, float) else (0, int(v), 0.0)
        preds[i] = Predicate(c, op, kind, 0, iv, fv)
    pay = (C.c_int32 * max(1, len(payload)))(*payload)
    ex = (Expr * max(1, len(exprs)))(*exprs)
    rc = lib().or_pipeline_run(C.byref(batch.desc), len(filters), preds, join.h if join else None, probe_key,
                               C.byref(build.desc) if build else None, len(payload), pay, len(exprs), ex, agg.h,
                               threads)
    if rc != 0:
        raise RuntimeError(_err())


def expr(result_type, program) -> Expr:
    """program items: ('col', i) | ('ci', v) | ('cf', v) | '+','-','*','/','>>','&'."""
    ops = {"+": 3, "-": 4, "*": 5, "/": 6, ">>": 7, "&": 8}
    e = Expr()
    e.result_type = result_type
    e.n_ops = len(program)
    for k, op in enumerate(program):
        if isinstance(op, str):
            e.ops[k] = ExprOp(ops[op], 0, 0, 0.0)
        elif op[0] == "col":
            e.ops[k] = ExprOp(0, op[1], 0, 0.0)
        elif op[0] == "ci":
            e.ops[k] = ExprOp(1, 0, int(op[1]), 0.0)
        else:
            e.ops[k] = ExprOp(2, 0, 0, float(op[1]))
    return e


# ---- generators --------------------------------------------------------------
def gen_starjoin_fact(n, seed=42, row0=0, threads=8):
    fk = np.empty(n, np.int32); qty = np.empty(n, np.int32)
    price = np.empty(n, DEC_DTYPE); disc = np.empty(n, np.float64)
    lib().or_gen_starjoin_fact(seed, row0, n, fk.ctypes.data, qty.ctypes.data, price.ctypes.data, disc.ctypes.data,
                               threads)
    return fk, qty, price, disc


def gen_starjoin_dim(n=1 << 22, seed=42):
    key = np.empty(n, np.int32); grp = np.empty(n, np.int32)
    lib().or_gen_starjoin_dim(seed, n, key.ctypes.data, grp.ctypes.data)
    return key, grp


def gen_groupby(n, seed=42, row0=0, ngroups=4096, threads=8):
    k = np.empty(n, np.int64); v = np.empty(n, np.int64); f = np.empty(n, np.float64); flag = np.empty(n, np.int32)
    lib().or_gen_groupby(seed, row0, n, ngroups, k.ctypes.data, v.ctypes.data, f.ctypes.data, flag.ctypes.data,
                         threads)
    return k, v, f, flag


def gen_highcard(n, seed=42, row0=0, threads=8):
    a = np.empty(n, np.int32); b = np.empty(n, np.int64); amt = np.empty(n, DEC_DTYPE); x = np.empty(n, np.float64)
    lib().or_gen_highcard(seed, row0, n, a.ctypes.data, b.ctypes.data, amt.ctypes.data, x.ctypes.data, threads)
    return a, b, amt, x


def i128_to_f64(hi, lo, scale) -> float:
    return lib().or_i128_to_f64(int(hi), int(lo) & ((1 << 64) - 1), scale)


def rle_decode(data: bytes, bit_width: int, count: int) -> np.ndarray:
    """DecodeRLEInt32 (rle.go): the hybrid stream's values (fewer than count when it ends early)."""
    buf = np.frombuffer(bytes(data), np.uint8) if len(data) else np.zeros(1, np.uint8)
    out = np.zeros(max(1, count), np.int32)
    n = lib().or_rle_decode(buf.ctypes.data, len(data), bit_width, count, out.ctypes.data)
    if n < 0:
        raise RuntimeError(_err())
    return out[:n].copy()


def page_decode(chunk, rows: int, out_dtype):
    """A column chunk (wadjet_b200._abi.wg_column_chunk) decoded on the CPU: (values, valid bool per row)."""
    out = np.zeros(max(1, rows), out_dtype)
    words = np.zeros(max(1, (rows + 63) // 64), np.uint64)
    if lib().or_page_decode(C.byref(chunk), out.ctypes.data, words.ctypes.data) != 0:
        raise RuntimeError(_err())
    valid = np.unpackbits(words.view(np.uint8), bitorder="little")[:rows].astype(bool)
    return out[:rows], valid


class StrGroupIndex:
    """String GROUP BY keys numbered as consumeBatchStrGroup numbers them
    (or_strindex_*, exec/aggregate.go:3038-3110): each distinct string takes the
    next group index at its first appearance, in row (selection) order across
    batches; a NULL string is the NULL-key group. `map` returns an INT32 column
    of group indexes and its validity, to aggregate like an int key."""

    def __init__(self):
        self.h = lib().or_strindex_new()
        self.n = 0

    def map_arrays(self, offs, raw, valid_words=None, sel=None, length=None):
        """Columnar form: offsets (uint32, len + 1), bytes (uint8), validity words."""
        n = len(offs) - 1 if length is None else length
        ids = np.zeros(max(n, 1), np.int32)
        o = np.ascontiguousarray(offs, np.uint32)
        b = np.ascontiguousarray(raw, np.uint8) if len(raw) else np.zeros(1, np.uint8)
        s = None if sel is None else np.ascontiguousarray(sel, np.uint32)
        self.n = lib().or_strindex_map(self.h, o.ctypes.data, b.ctypes.data, _ptr(valid_words), n, _ptr(s),
                                       0 if s is None else len(s), ids.ctypes.data)
        return ids[:n]

    def map(self, values, valid=None, sel=None):
        enc = [b"" if (valid is not None and not valid[i]) else v for i, v in enumerate(values)]
        offs = np.zeros(len(enc) + 1, np.uint32)
        if enc:
            offs[1:] = np.cumsum([len(v) for v in enc])
        raw = np.frombuffer(b"".join(enc), np.uint8)
        w = None if valid is None else pack_validity(np.asarray(valid, bool))
        ids = self.map_arrays(offs, raw, w, sel)
        return ids, (None if valid is None else np.asarray(valid, bool))

    @property
    def strings(self) -> list:
        """Every string by its group index (fetched once; later calls only add new ones)."""
        out = self.__dict__.setdefault("_strings", [])
        for i in range(len(out), self.n):
            ln = lib().or_strindex_get(self.h, i, None, 0)
            buf = np.zeros(max(ln, 1), np.uint8)
            lib().or_strindex_get(self.h, i, buf.ctypes.data, ln)
            out.append(buf[:ln].tobytes())
        return list(out)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_strindex_free(self.h)
            self.h = None
