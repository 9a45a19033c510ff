"""The CPU oracle against the reference's own known-answer tests (golden fixtures).

These pin the oracle before it is trusted as the checker of the GPU path.
"""
import json
import os

import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import dec_array

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))

NP = {1: np.int32, 2: np.int64, 3: np.float32, 4: np.float64, 7: np.int64, 8: np.int64, 11: np.int64,
      12: np.int32, 13: np.int32, 14: np.int64, 16: np.int32}


def col_array(t, values):
    if t == 17:
        return dec_array(values)
    return np.array(values, dtype=NP[t])


def valid_of(n, nulls):
    if not nulls:
        return None
    v = np.ones(n, bool)
    v[nulls] = False
    return v


@pytest.mark.parametrize("case", GOLD["filters"], ids=lambda c: c["ref"])
def test_filter_known_answers(case):
    data = col_array(case["type"], case["values"])
    got = ob.filter_(case["type"], data, valid_of(len(data), case["nulls"]), case["op"], case["const"],
                     sel=case["sel"])
    assert got.tolist() == case["expect"]


@pytest.mark.parametrize("case", GOLD["accumulators"], ids=lambda c: c["ref"])
def test_accumulator_known_answers(case):
    t = case["type"]
    data = col_array(t, case["values"])
    agg = ob.Agg([], [(case["func"], -1 if case["star"] else 0, 0)])
    agg.consume(ob.HostBatch([(t, data, valid_of(len(data), case["nulls"]), 2 if t == 17 else 0)], sel=case["sel"]))
    e = agg.export()
    exp = case["expect"]
    if "count" in exp:
        assert e["count"][0, 0] == exp["count"]
    if "i64" in exp:
        assert e["i64"][0, 0] == exp["i64"]
    if "f64" in exp:
        assert e["f64"][0, 0] == exp["f64"]
    if "dec" in exp:
        assert int(e["dec"][0, 0]["lo"]) == exp["dec"] and int(e["dec"][0, 0]["hi"]) == 0
    if "has" in exp:
        assert e["has"][0, 0] == exp["has"]
    if "final" in exp:
        out = agg.emit([np.float64])
        assert out[0][1][0] and out[0][0][0] == exp["final"]


def test_decimal_known_answers():
    d = GOLD["decimal"]
    for v, hi, lo in d["from"]:
        a = dec_array([v])[0]
        assert int(a["hi"]) == hi and int(a["lo"]) == lo
    # Add and Less through one-group aggregates (SUM / MIN over DECIMAL)
    for (ah, al), (bh, bl), (ch, cl) in d["add"]:
        vals = np.zeros(2, ob.DEC_DTYPE)
        vals[0] = (ah, al)
        vals[1] = (bh, bl)
        agg = ob.Agg([], [(0, 0, 0)])
        agg.consume(ob.HostBatch([(17, vals, None, 0)]))
        got = agg.export()["dec"][0, 0]
        assert (int(got["hi"]), int(got["lo"])) == (ch, cl)
    for (ah, al), (bh, bl), less in d["less"]:
        vals = np.zeros(2, ob.DEC_DTYPE)
        vals[0] = (ah, al)
        vals[1] = (bh, bl)
        agg = ob.Agg([], [(2, 0, 0)])
        agg.consume(ob.HostBatch([(17, vals, None, 0)]))
        got = agg.export()["dec"][0, 0]
        want = (ah, al) if less else (bh, bl)
        if (ah, al) == (bh, bl):
            want = (ah, al)
        assert (int(got["hi"]), int(got["lo"])) == want
    for hi, lo, scale, want in d["to_f64"]:
        assert abs(ob.i128_to_f64(hi, lo, scale) - want) <= 1e-3 * max(1.0, abs(want))


def test_groupby_known_answer():
    for c in GOLD["groupby"]:
        keys = np.array(c["keys"], np.int64)
        amt = np.array(c["amount"], np.float64)
        agg = ob.Agg([0], [(0, 1, 0), (1, 1, 0)])
        agg.consume(ob.HostBatch([(2, keys, None, 0), (4, amt, None, 0)]))
        e = agg.export()
        got = {str(k): [e["f64"][0, i], e["count"][1, i]] for i, k in enumerate(e["keys"][0])}
        assert got == c["expect"]


@pytest.mark.parametrize("case", GOLD["string_groupby"], ids=lambda c: c["ref"])
def test_string_groupby_known_answer(case):
    """consumeBatchStrGroup: group indexes by first appearance, NULL its own group
    (distinct from the one-byte string \x01), accumulated across batches."""
    idx = ob.StrGroupIndex()
    agg = ob.Agg([0], [(1, -1, 0), (0, 1, 0)])
    for rows in case["batches"]:
        keys = [b"" if k is None else k.encode() for k, _ in rows]
        valid = np.array([k is not None for k, _ in rows], bool)
        ids, ok = idx.map(keys, valid)
        v = np.array([x for _, x in rows], np.int64)
        agg.consume(ob.HostBatch([(1, ids, ok, 0), (2, v, None, 0)]))
    e = agg.export()
    strs = idx.strings
    got = sorted([[strs[int(e["keys"][0, i])].decode() if e["key_valid"][0, i] else None,
                   int(e["count"][0, i]), int(e["i64"][1, i])] for i in range(e["count"].shape[1])],
                 key=lambda r: (r[0] is None, r[0] or ""))
    want = sorted(case["expect"], key=lambda r: (r[0] is None, r[0] or ""))
    assert got == want
    # first-appearance numbering
    first = []
    for rows in case["batches"]:
        for k, _ in rows:
            if k is not None and k.encode() not in first:
                first.append(k.encode())
    assert strs == first


def test_join_known_answer():
    for c in GOLD["joins"]:
        j = ob.Join()
        j.append(2, np.array(c["build_keys"], np.int64))
        pr, br = j.probe(2, np.array(c["probe_keys"], np.int64))
        assert sorted(zip(pr.tolist(), br.tolist())) == sorted(map(tuple, c["expect_pairs"]))


@pytest.mark.parametrize("case", GOLD["packed_layout"], ids=lambda c: c[0])
def test_packed_layout_eligibility(case):
    name, types, eligible = case
    cols = [(t, np.zeros(4, NP.get(t, np.int64)), None, 0) for t in types]
    agg = ob.Agg(list(range(len(types))), [(1, -1, 0)])
    try:
        agg.consume(ob.HostBatch(cols))
        ok = True
    except RuntimeError:
        ok = False
    # a single int key is eligible for the int-key path; the packed path needs >= 2 columns
    if len(types) == 1:
        assert ok
    else:
        assert ok == eligible


def test_extreme_packed_keys_are_real_groups():
    keys = GOLD["extreme_keys"]["keys"]
    a = np.array([k[0] for k in keys], np.uint64).view(np.int64)
    b = np.array([k[1] for k in keys], np.uint64).view(np.int64)
    agg = ob.Agg([0, 1], [(1, -1, 0)])
    agg.consume(ob.HostBatch([(2, a, None, 0), (2, b, None, 0)]))
    e = agg.export()
    assert e["keys"].shape[1] == len(keys)
    assert sorted(zip(e["keys"][0].tolist(), e["keys"][1].tolist())) == sorted(zip(a.tolist(), b.tolist()))


def test_packed_round_trip_values():
    rt = GOLD["round_trip"]
    i64 = np.array(rt["i64"], np.int64)
    i32 = np.array(rt["i32"] + rt["i32"][:2], np.int32)[: len(i64)]
    agg = ob.Agg([0, 1], [(1, -1, 0)])
    agg.consume(ob.HostBatch([(1, i32, None, 0), (2, i64, None, 0)]))
    e = agg.export()
    assert sorted(zip(e["keys"][0].tolist(), e["keys"][1].tolist())) == sorted(zip(i32.tolist(), i64.tolist()))


@pytest.mark.parametrize("case", GOLD["rle"], ids=lambda c: c["ref"])
def test_rle_hybrid_known_answers(case):
    """The oracle's RLE / bit-packed hybrid decoder on the reference's rle_test.go vectors."""
    got = ob.rle_decode(bytes(case["data"]), case["bit_width"], case["count"])
    assert got.tolist() == case["expect"]


@pytest.mark.parametrize("bw", [1, 3, 7, 12, 20, 32])
def test_page_encoder_round_trips_through_the_oracle(bw):
    """wadjet_b200.pages writes hybrid streams the oracle's decoder reads back, runs of
    repeated values and bit-packed stretches alike."""
    from wadjet_b200 import pages
    rng = np.random.default_rng(bw)
    top = (1 << bw) - 1
    v = rng.integers(0, top + 1, 5000, dtype=np.int64)
    v[1000:1400] = top          # a long repeated run
    v[2000:2005] = 0            # a short one, bit-packed
    enc = pages.encode_hybrid(v, bw)
    np.testing.assert_array_equal(ob.rle_decode(enc, bw, len(v)), v.astype(np.int32))


def test_page_decode_oracle_plain_dictionary_and_nulls():
    """The oracle's page decode: PLAIN and dictionary pages, NULL rows from the levels,
    DECIMAL INT64 widened to Int128 (Int128From)."""
    from tests.helpers import dec_array
    from wadjet_b200 import pages
    rng = np.random.default_rng(9)
    n = 3000
    vals = rng.integers(-50, 50, n).astype(np.int64)
    valid = rng.random(n) > 0.2
    for dictionary in (False, True):
        ch = pages.chunk(vals, 2, valid, page_rows=1000, dictionary=dictionary)
        out, ok = ob.page_decode(ch.to_c(), n, np.int64)
        np.testing.assert_array_equal(ok, valid)
        np.testing.assert_array_equal(out[valid], vals[valid])
        assert (out[~valid] == 0).all()
    dec = dec_array(vals)
    ch = pages.chunk(dec, 17, None, page_rows=700, dictionary=True, scale=2)
    out, ok = ob.page_decode(ch.to_c(), n, dec.dtype)
    assert ok.all()
    np.testing.assert_array_equal(out["lo"], dec["lo"])
    np.testing.assert_array_equal(out["hi"], dec["hi"])
