"""Write tests/golden/known_answers.json: the reference's own known-answer tests
for the filter → hash-join → hash-aggregate path, restated as data.

The reference is Go and cannot run here, so each case below transcribes the
inputs and the expected outputs of one reference test (cited as file:line in
the Wadjet tree). String keys in the reference's join tests and in the
integer-key aggregate case are restated as integer keys; the expected row
counts and sums are unchanged by that renaming. The string GROUP BY cases keep
their strings.

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os

I32, I64, F32, F64, TS, IPV4, MAC, PORT, PROTO, DUR, DATE, DEC = 1, 2, 3, 4, 7, 8, 11, 12, 13, 14, 16, 17
EQ, NE, LT, LE, GT, GE = range(6)
SUM, COUNT, MIN, MAX, AVG = range(5)

# ---- filter kernels: (ref, type, values, null rows, sel, op, const, expected selection) -------------
FILTERS = [
    ("internal/engine/exec/kernel/kernel_test.go:144", I64, [10, 20, 30, 40, 50], [], None, GT, 25, [2, 3, 4]),
    ("internal/engine/exec/kernel/kernel_test.go:161", F64, [1.0, 2.5, 3.0, 0.5], [], None, LE, 2.5, [0, 1, 3]),
    ("internal/engine/exec/kernel/kernel_test.go:181", I64, [10, 20, 30, 40, 50], [], [0, 2, 4], GT, 15, [2, 4]),
    ("internal/engine/exec/kernel/kernel_test.go:192", I64, [10, 20, 30], [1], None, GT, 5, [0, 2]),
    ("internal/engine/exec/kernel/agg_test.go:629 (OpEq)", I64, [10, 20, 30], [], None, EQ, 20, [1]),
    ("internal/engine/exec/kernel/agg_test.go:629 (OpNe)", I64, [10, 20, 30], [], None, NE, 20, [0, 2]),
    ("internal/engine/exec/kernel/agg_test.go:629 (OpLt)", I64, [10, 20, 30], [], None, LT, 20, [0]),
    ("internal/engine/exec/kernel/agg_test.go:629 (OpLe)", I64, [10, 20, 30], [], None, LE, 20, [0, 1]),
    ("internal/engine/exec/kernel/agg_test.go:629 (OpGt)", I64, [10, 20, 30], [], None, GT, 20, [2]),
    ("internal/engine/exec/kernel/agg_test.go:629 (OpGe)", I64, [10, 20, 30], [], None, GE, 20, [1, 2]),
    ("internal/engine/exec/kernel/agg_test.go:655", F32, [1.0, 2.0, 3.0], [], None, GT, 1.5, [1, 2]),
    ("internal/engine/exec/kernel/agg_test.go:665", I32, [10, 20, 30], [], None, EQ, 20, [1]),
    ("internal/engine/exec/kernel/agg_test.go:829", PORT, [80, 443, 22], [], None, EQ, 443, [1]),
    ("internal/engine/exec/kernel/agg_test.go:843", DUR, [100, 200, 300], [], None, GT, 150, [1, 2]),
    ("internal/engine/exec/kernel/agg_test.go:857", DATE, [100, 200, 300], [], None, LT, 200, [0]),
    # IPv4 192.168.1.1 / 10.0.0.1 stored as their uint32 value in Int64Data (compare.go:158, parseIPv4ToInt64)
    ("internal/engine/exec/kernel/agg_test.go:797", IPV4, [3232235777, 167772161], [], None, EQ, 3232235777, [0]),
    # MAC aa:bb:cc:dd:ee:ff / 00:11:22:33:44:55 as 48-bit values (parseMACToInt64)
    ("internal/engine/exec/kernel/agg_test.go:813", MAC, [0xAABBCCDDEEFF, 0x001122334455], [], None, EQ,
     0xAABBCCDDEEFF, [0]),
]

# ---- accumulators over one column (scalar aggregate, no GROUP BY) ---------------------------------------
# (ref, type, values, null rows, sel, func, expected {count, i64|f64|dec, final})
ACCUMULATORS = [
    ("internal/engine/exec/kernel/kernel_test.go:40", I64, [10, 20, 30, 40, 50], [], None, SUM, {"count": 5, "i64": 150}),
    ("internal/engine/exec/kernel/kernel_test.go:53", I64, [10, 20, 30, 40, 50], [1, 3], None, SUM, {"count": 3, "i64": 90}),
    ("internal/engine/exec/kernel/kernel_test.go:66", F64, [1.5, 2.5, 3.0], [], None, SUM, {"count": 3, "f64": 7.0}),
    ("internal/engine/exec/kernel/kernel_test.go:79", I64, [10, 20, 30, 40, 50], [], [0, 2, 4], SUM, {"count": 3, "i64": 90}),
    ("internal/engine/exec/kernel/kernel_test.go:93", I64, [10, 20, 30], [], None, SUM, {"i64": 60}),
    ("internal/engine/exec/kernel/kernel_test.go:105 (min)", I64, [30, 10, 50, 20, 40], [], None, MIN, {"i64": 10}),
    ("internal/engine/exec/kernel/kernel_test.go:105 (max)", I64, [30, 10, 50, 20, 40], [], None, MAX, {"i64": 50}),
    ("internal/engine/exec/kernel/kernel_test.go:122 (col)", I64, [10, 20, 30], [1], None, COUNT, {"count": 2}),
    ("internal/engine/exec/kernel/kernel_test.go:122 (star)", I64, [10, 20, 30], [1], None, -COUNT - 1, {"count": 3}),
    ("internal/engine/exec/kernel/agg_test.go:44", I32, [10, 20, 30], [], None, SUM, {"i64": 60}),
    ("internal/engine/exec/kernel/agg_test.go:59", F64, [1.5, 2.5, 3.0], [], None, SUM, {"f64": 7.0}),
    ("internal/engine/exec/kernel/agg_test.go:74", F32, [1.0, 2.0, 3.0], [], None, SUM, {"f64": 6.0}),
    ("internal/engine/exec/kernel/agg_test.go:92", DEC, [100, 200, 300], [], None, SUM, {"count": 3, "dec": 600, "final": 6.0}),
    ("internal/engine/exec/kernel/agg_test.go:110", I64, [10, 20, 30], [1], None, SUM, {"count": 2, "i64": 40}),
    ("internal/engine/exec/kernel/agg_test.go:134", I32, [30, 10, 50], [], None, MIN, {"i64": 10}),
    ("internal/engine/exec/kernel/agg_test.go:149", F64, [3.0, 1.5, 2.5], [], None, MIN, {"f64": 1.5}),
    ("internal/engine/exec/kernel/agg_test.go:161", F32, [3.0, 1.5, 2.5], [], None, MIN, {"f64": 1.5}),
    ("internal/engine/exec/kernel/agg_test.go:176", DEC, [300, 100, 200], [], None, MIN, {"has": 1, "dec": 100, "final": 1.0}),
    ("internal/engine/exec/kernel/agg_test.go:194", I64, [30, 10, 50], [1], None, MIN, {"i64": 30}),
    ("internal/engine/exec/kernel/agg_test.go:217", I32, [30, 10, 50], [], None, MAX, {"i64": 50}),
    ("internal/engine/exec/kernel/agg_test.go:232", F64, [3.0, 1.5, 2.5], [], None, MAX, {"f64": 3.0}),
    ("internal/engine/exec/kernel/agg_test.go:244", F32, [3.0, 1.5, 2.5], [], None, MAX, {"f64": 3.0}),
    ("internal/engine/exec/kernel/agg_test.go:259", DEC, [100, 300, 200], [], None, MAX, {"has": 1, "dec": 300, "final": 3.0}),
    ("internal/engine/exec/kernel/agg_test.go:347", DEC, [1000], [], None, SUM, {"count": 1, "final": 10.0}),
    ("internal/engine/exec/kernel/agg_test.go:364", DEC, [400, 600], [], None, AVG, {"count": 2, "final": 5.0}),
    ("internal/engine/exec/kernel/agg_test.go:380", I32, [10, 20, 30], [], None, SUM, {"i64": 60}),
    ("internal/engine/exec/kernel/agg_test.go:393", F32, [1.0, 2.0, 3.0], [], None, SUM, {"f64": 6.0}),
    ("internal/engine/exec/kernel/agg_test.go:406", DEC, [100, 200, 300], [], None, SUM, {"count": 3}),
    ("internal/engine/exec/kernel/agg_test.go:422", DEC, [100, 200, 300], [], [0, 2], SUM, {"count": 2, "dec": 400}),
    ("internal/engine/exec/kernel/agg_test.go:433", DEC, [100, 200, 300], [1], None, SUM, {"count": 2, "dec": 400}),
    ("internal/engine/exec/kernel/agg_test.go:452", I64, [10, 20, 30], [1], None, COUNT, {"count": 2}),
    ("internal/engine/exec/kernel/agg_test.go:462", I64, [10, 20, 30, 40], [1], [0, 1, 3], COUNT, {"count": 2}),
    ("internal/engine/exec/kernel/agg_test.go:473", I64, [10, 20, 30], [], None, COUNT, {"count": 3}),
    ("internal/engine/exec/kernel/agg_test.go:483", I64, [10, 20, 30], [], [0, 2], COUNT, {"count": 2}),
    ("internal/engine/exec/kernel/agg_test.go:496", I64, [10, 20, 30, 40, 50], [2], [0, 2, 4], SUM, {"count": 2, "i64": 60}),
]

# ---- Int128 (internal/engine/batch/decimal_test.go) ----------------------------------------------------
DECIMAL = {
    "from": [  # decimal_test.go:8: Int128From(v) = {Hi, Lo}
        [0, 0, 0], [1, 0, 1], [-1, -1, 2**64 - 1], [12345, 0, 12345], [-12345, -1, 2**64 - 12345],
        [2**63 - 1, 0, 2**63 - 1],
    ],
    "add": [  # decimal_test.go:30 (100+50) plus carry cases of decimal.go:78
        [[0, 100], [0, 50], [0, 150]],
        [[0, 2**64 - 1], [0, 1], [1, 0]],
        [[-1, 2**64 - 1], [0, 1], [0, 0]],
        [[0, 100], [-1, 2**64 - 50], [0, 50]],
    ],
    "less": [  # decimal_test.go:50
        [[0, 100], [0, 200], True], [[0, 200], [0, 100], False], [[-1, 2**64 - 50], [0, 100], True],
        [[0, 100], [0, 100], False],
    ],
    "to_f64": [  # decimal_test.go:99 (within 0.001) and the Hi/Lo branches of decimal.go:39
        [0, 12345, 2, 123.45], [-1, 2**64 - 9999, 2, -99.99], [0, 1000, 2, 10.0], [1, 0, 0, 18446744073709551616.0],
    ],
}

# ---- grouped aggregate: exec_test.go:39 TestHashAggregate, string keys a,b restated as 1,2 -------------
GROUPBY = [{
    "ref": "internal/engine/exec/exec_test.go:39",
    "keys": [1, 2, 1, 2], "amount": [10.0, 20.0, 30.0, 40.0],
    "aggs": [[SUM, "amount"], [COUNT, "amount"]],
    "expect": {"1": [40.0, 2], "2": [60.0, 2]},
}]

# ---- string GROUP BY keys (consumeBatchStrGroup, aggregate.go:3038) --------------------------------------
# batches of (key or None, value); expect: key (None = the NULL group) -> [COUNT(*), SUM(v)]
STRING_GROUPBY = [
    {"ref": "internal/engine/exec/aggregate_null_group_test.go:226",
     "batches": [[["a", 1], [None, 10], ["b", 2], [None, 20]],
                 [[None, 30], ["a", 3], ["\x01", 100]]],
     "expect": [["a", 2, 4], ["b", 1, 2], ["\x01", 1, 100], [None, 3, 60]]},
    # exec_test.go:39 TestHashAggregate with its string keys; SUM(amount) of float64 restated as int64
    {"ref": "internal/engine/exec/exec_test.go:39",
     "batches": [[["a", 10], ["b", 20], ["a", 30], ["b", 40]]],
     "expect": [["a", 2, 40], ["b", 2, 60]]},
]

# ---- inner join: join_test.go:10 TestHashJoin_Inner, alice=1 bob=2 carol=3 unknown=4 -------------------
JOINS = [{
    "ref": "internal/engine/exec/join_test.go:10",
    "probe_keys": [1, 2, 1, 4], "probe_amount": [100.0, 200.0, 150.0, 50.0],
    "build_keys": [1, 2, 3],
    "expect_pairs": [[0, 0], [1, 1], [2, 0]],
}]

# ---- packed-key eligibility: packed_hash_test.go:175 TestBuildPackedLayoutEligibility ---------------
PACKED_LAYOUT = [
    ["single column declines", [I64], False],
    ["two int64 = 16B exactly", [I64, I64], True],
    ["int64+int32 = 12B", [I64, I32], True],
    ["three int32 = 12B", [I32, I32, I32], True],
    ["four int32 = 16B exactly", [I32, I32, I32, I32], True],
    ["int32,int64,int32 = 16B needs widest-first", [I32, I64, I32], True],
    ["two int64 + int32 = 20B declines", [I64, I64, I32], False],
    ["five int32 = 20B declines", [I32, I32, I32, I32, I32], False],
    ["float column declines", [I64, F64], False],
    ["network types pack", [IPV4, MAC], True],
    ["port+protocol+date+int32", [PORT, PROTO, DATE, I32], True],
]

# ---- packed keys that collide with table sentinels: packed_hash_test.go:74 ------------------------------
U64MAX = 2**64 - 1
EXTREME_KEYS = {
    "ref": "internal/engine/exec/packed_hash_test.go:74",
    "keys": [[0, 0], [U64MAX, U64MAX], [0, U64MAX], [U64MAX, 0], [1, 0], [0, 1]],
}

# ---- packed-key round trip values: packed_hash_test.go:235 ----------------------------------------------
ROUND_TRIP = {
    "ref": "internal/engine/exec/packed_hash_test.go:235",
    "i64": [0, 1, -1, 2**63 - 1, -2**63, 1 << 40, -(1 << 40), 0xFFFFFFFF, 0xFFFFFFFFFFFF],
    "i32": [0, 1, -1, 2**31 - 1, -2**31, 1 << 30, -(1 << 30)],
}


# ---- Parquet RLE / bit-packed hybrid: internal/storage/parquet/rle_test.go -----------------------------
def _le16(*vals):
    out = []
    for v in vals:
        out += [v & 0xFF, v >> 8]
    return out


def _varint(v):
    out = []
    while v >= 0x80:
        out.append((v & 0x7F) | 0x80)
        v >>= 7
    return out + [v]


# (ref, stream bytes, bit width, count, expected values). Bit-packed vectors of
# TestDecodeBitPacked are wrapped as one bit-packed run (header (groups << 1) | 1)
# of the stream the hybrid decoder reads.
RLE = [
    ("internal/storage/parquet/rle_test.go:17 (1bit_8values)", [3, 0b10110010], 1, 8, [0, 1, 0, 0, 1, 1, 0, 1]),
    ("internal/storage/parquet/rle_test.go:23 (2bit_4values)", [3, 0b11100100, 0, 0, 0, 0, 0, 0, 0][:3], 2, 4,
     [0, 1, 2, 3]),
    ("internal/storage/parquet/rle_test.go:47 (0bit)", [3], 0, 5, [0, 0, 0, 0, 0]),
    ("internal/storage/parquet/rle_test.go:52 (8bit)", [3, 10, 20, 30, 0, 0, 0, 0, 0], 8, 3, [10, 20, 30]),
    ("internal/storage/parquet/rle_test.go:57 (16bit)", [3] + _le16(1000, 2000) + [0] * 12, 16, 2, [1000, 2000]),
    ("internal/storage/parquet/rle_test.go:91 (TestRLERun)", [20, 42], 8, 10, [42] * 10),
    ("internal/storage/parquet/rle_test.go:112 (TestRLERunMultiByte)", [10, 0x2C, 0x01], 16, 5, [300] * 5),
    ("internal/storage/parquet/rle_test.go:134 (TestRLEBitPackedRun)", [3, 10, 20, 30, 40, 50, 60, 70, 80], 8, 8,
     [10, 20, 30, 40, 50, 60, 70, 80]),
    ("internal/storage/parquet/rle_test.go:154 (TestRLEMixed)", [8, 0, 3, 0x55], 1, 12,
     [0, 0, 0, 0, 1, 0, 1, 0, 1, 0, 1, 0]),
    ("internal/storage/parquet/rle_test.go:217 (TestRLEBitWidth1)", _varint(100 << 1) + [1], 1, 100, [1] * 100),
    ("internal/storage/parquet/rle_test.go:239 (TestRLEEmpty)", [], 8, 0, []),
]


def main() -> None:
    out = {
        "filters": [dict(ref=r, type=t, values=v, nulls=n, sel=s, op=o, const=c, expect=e)
                    for r, t, v, n, s, o, c, e in FILTERS],
        "accumulators": [dict(ref=r, type=t, values=v, nulls=n, sel=s,
                              func=(COUNT if f < 0 else f), star=(f < 0), expect=e)
                         for r, t, v, n, s, f, e in ACCUMULATORS],
        "decimal": DECIMAL,
        "groupby": GROUPBY,
        "string_groupby": STRING_GROUPBY,
        "joins": JOINS,
        "packed_layout": PACKED_LAYOUT,
        "extreme_keys": EXTREME_KEYS,
        "round_trip": ROUND_TRIP,
        "rle": [dict(ref=r, data=d, bit_width=b, count=c, expect=e) for r, d, b, c, e in RLE],
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path)


if __name__ == "__main__":
    main()
