"""The reference's known-answer tests through the GPU library (C ABI)."""
import json
import os

import numpy as np
import pytest

from tests.helpers import dec_array

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))
NP = {1: np.int32, 2: np.int64, 3: np.float32, 4: np.float64, 7: np.int64, 8: np.int64, 11: np.int64,
      12: np.int32, 13: np.int32, 14: np.int64, 16: np.int32}


def col(t, values, nulls=(), scale=0):
    import wadjet_b200 as wg
    data = dec_array(values) if t == 17 else np.array(values, dtype=NP[t])
    valid = None
    if nulls:
        valid = np.ones(len(data), bool)
        valid[list(nulls)] = False
    return wg.Column(t, data, valid, scale)


@pytest.mark.parametrize("case", GOLD["filters"], ids=lambda c: c["ref"])
def test_filter_known_answers(ctx, case):
    import wadjet_b200 as wg
    f = wg.KernelFilter(ctx, 0, case["op"], case["const"])
    out = f.execute(wg.Batch([col(case["type"], case["values"], case["nulls"])], sel=case["sel"]))
    assert (out.tolist() if out is not None else []) == case["expect"]
    f.close()


@pytest.mark.parametrize("case", GOLD["accumulators"], ids=lambda c: c["ref"])
def test_accumulator_known_answers(ctx, case):
    import wadjet_b200 as wg
    t = case["type"]
    agg = wg.HashAggregate(ctx, [], [wg.AggColumn(case["func"], -1 if case["star"] else 0)])
    agg.consume(wg.Batch([col(t, case["values"], case["nulls"], 2 if t == 17 else 0)], sel=case["sel"]))
    agg.finalize()
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
        page = agg.next()
        assert page[0][1][0] and page[0][0][0] == exp["final"]
    agg.close()


def test_groupby_known_answer(ctx):
    import wadjet_b200 as wg
    for c in GOLD["groupby"]:
        agg = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, 1)])
        agg.consume(wg.Batch([col(2, c["keys"]), col(4, c["amount"])]))
        agg.finalize()
        rows = agg.collect()
        got = {str(k): [s, n] for k, s, n in zip(rows[0][0].tolist(), rows[1][0].tolist(), rows[2][0].tolist())}
        assert got == c["expect"]
        agg.close()


@pytest.mark.parametrize("case", GOLD["string_groupby"], ids=lambda c: c["ref"])
def test_string_groupby_known_answer(ctx, case):
    import wadjet_b200 as wg
    agg = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_SUM, 1)])
    for rows in case["batches"]:
        agg.consume(wg.Batch([wg.Column.strings([k for k, _ in rows]),
                              wg.Column(2, np.array([x for _, x in rows], np.int64))]))
    agg.finalize()
    out = agg.collect()
    got = sorted([[out[0][0][i] if out[0][1][i] else None, int(out[1][0][i]), int(out[2][0][i])]
                  for i in range(len(out[0][0]))], key=lambda r: (r[0] is None, r[0] or ""))
    assert got == sorted(case["expect"], key=lambda r: (r[0] is None, r[0] or ""))
    agg.close()


def test_join_known_answer(ctx):
    import wadjet_b200 as wg
    for c in GOLD["joins"]:
        j = wg.HashJoin(ctx, 0, 0)
        j.build([wg.Batch([col(2, c["build_keys"])])])
        pairs = []
        for pr, br in j.probe(wg.Batch([col(2, c["probe_keys"]), col(4, c["probe_amount"])])):
            pairs += list(zip(pr.tolist(), br.tolist()))
        assert sorted(pairs) == sorted(map(tuple, c["expect_pairs"]))
        j.close()


def test_extreme_packed_keys_are_real_groups(ctx):
    import wadjet_b200 as wg
    keys = GOLD["extreme_keys"]["keys"]
    a = np.array([k[0] for k in keys], np.uint64).view(np.int64)
    b = np.array([k[1] for k in keys], np.uint64).view(np.int64)
    agg = wg.HashAggregate(ctx, [0, 1], [wg.AggColumn(wg.AGG_COUNT, -1)])
    agg.consume(wg.Batch([wg.Column(2, a), wg.Column(2, b)]))
    agg.finalize()
    e = agg.export()
    assert sorted(zip(e["keys"][0].tolist(), e["keys"][1].tolist())) == sorted(zip(a.tolist(), b.tolist()))
    assert e["count"][0].tolist() == [1] * len(keys)
    agg.close()


def test_packed_round_trip_values(ctx):
    import wadjet_b200 as wg
    rt = GOLD["round_trip"]
    i64 = np.array(rt["i64"], np.int64)
    i32 = np.array(rt["i32"] + rt["i32"][:2], np.int32)[: len(i64)]
    agg = wg.HashAggregate(ctx, [0, 1], [wg.AggColumn(wg.AGG_COUNT, -1)])
    agg.consume(wg.Batch([wg.Column(1, i32), wg.Column(2, i64)]))
    agg.finalize()
    e = agg.export()
    assert sorted(zip(e["keys"][0].tolist(), e["keys"][1].tolist())) == sorted(zip(i32.tolist(), i64.tolist()))
    agg.close()
