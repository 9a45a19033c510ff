"""Parity at the sizes the measurements are quoted on, group by group.

- Star join at 2^28 fact rows (the headline): all 1000 groups against the oracle
  over the same 2^28 rows (the oracle's Pipeline.Run on every host thread).
- High-cardinality GROUP BY at 2^26 rows (~42M groups, the two-level mode with
  its 2^15 buckets): every group against the oracle.
- High-cardinality GROUP BY at 2^28 rows (~65.9M groups): the resident result
  equals, bit for bit, the result under an 8 GB HBM cap (the pinned-host spill).
- Batched mode: all 512 queries of the configured workload at full size
  (up to 10^7 rows and 10^6 groups each), each against its own oracle run.

Parallel = serial: a partition of the work must not change any group
(partitioned_agg_test.go:91, packed_agg_test.go:278).
"""
import os

import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import DEC_DTYPE, assert_groups_equal

pytestmark = pytest.mark.gpu

I32, I64, F64, DEC = 1, 2, 4, 17
THREADS = os.cpu_count() or 8


def _free():
    import gc
    import torch
    gc.collect()
    torch.cuda.empty_cache()


def test_starjoin_2p28_every_group_matches_oracle(ctx):
    import wadjet_b200 as wg
    from wadjet_b200 import synth
    n, nd = 1 << 28, 1 << 22
    fk, qty, price, disc = synth.starjoin_fact(ctx, n)
    key, grp = synth.starjoin_dim(ctx)
    j = wg.HashJoin(ctx, 0, 0, payload=[1], build_row_hint=nd)
    j.build([wg.Batch([wg.Column(I32, key), wg.Column(I32, grp)])], device=True)
    expr = wg.Expr(F64, [wg.Expr.col(2), wg.Expr.const_f(1.0), wg.Expr.col(3), "-", "*"])
    aggs = [wg.AggColumn(wg.AGG_SUM, 5), wg.AggColumn(wg.AGG_SUM, 2), wg.AggColumn(wg.AGG_COUNT, -1)]
    g = wg.HashAggregate(ctx, [4], aggs, ndv_hint=1000)
    wg.run_pipeline(ctx, wg.Batch([wg.Column(I32, fk), wg.Column(I32, qty), wg.Column(DEC, price, scale=2),
                                   wg.Column(F64, disc)]), g, filters=[(1, wg.OP_GT, 10)], join=j, exprs=[expr],
                    device=True)
    g.finalize()
    got = g.export()
    g.close()
    j.close()
    del fk, qty, price, disc, key, grp
    _free()
    hfk, hqty, hprice, hdisc = ob.gen_starjoin_fact(n, threads=THREADS)
    hkey, hgrp = ob.gen_starjoin_dim(nd)
    oj = ob.Join(nd)
    oj.append(I32, hkey)
    o = ob.Agg([4], [(0, 5, 0), (0, 2, 0), (1, -1, 0)])
    ob.pipeline(ob.HostBatch([(I32, hfk, None, 0), (I32, hqty, None, 0), (DEC, hprice.view(DEC_DTYPE), None, 2),
                              (F64, hdisc, None, 0)]), o, filters=[(1, wg.OP_GT, 10)], join=oj, probe_key=0,
                build=ob.HostBatch([(I32, hkey, None, 0), (I32, hgrp, None, 0)]), payload=[1],
                exprs=[ob.expr(F64, [("col", 2), ("cf", 1.0), ("col", 3), "-", "*"])], threads=THREADS)
    want = o.export()
    assert got["keys"].shape[1] == 1000
    assert_groups_equal(got, want, ["sum_f", "sum_d", "count"])


def _highcard(ctx, n, hint, cap=0):
    import wadjet_b200 as wg
    from wadjet_b200 import synth
    c = ctx if not cap else wg.Context(0, hbm_budget=cap, pinned_spill=24 << 30)
    a, b, amt, x = synth.highcard(c, n)
    aggs = [wg.AggColumn(wg.AGG_SUM, 2), wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_MIN, 3),
            wg.AggColumn(wg.AGG_MAX, 3)]
    g = wg.HashAggregate(c, [0, 1], aggs, ndv_hint=hint)
    wg.run_pipeline(c, wg.Batch([wg.Column(I32, a), wg.Column(I64, b), wg.Column(DEC, amt, scale=2),
                                 wg.Column(F64, x)]), g, device=True)
    g.finalize()
    out = g.export()
    peak = c.ledger()["peak"]
    g.close()
    del a, b, amt, x
    if cap:
        c.close()
    _free()
    return out, peak


def test_highcard_2p26_every_group_matches_oracle(ctx):
    n = 1 << 26
    got, _ = _highcard(ctx, n, 1 << 26)
    ha, hb, hamt, hx = ob.gen_highcard(n, threads=THREADS)
    o = ob.Agg([0, 1], [(0, 2, 0), (1, -1, 0), (2, 3, 0), (3, 3, 0)])
    ob.pipeline(ob.HostBatch([(I32, ha, None, 0), (I64, hb, None, 0), (DEC, hamt.view(DEC_DTYPE), None, 2),
                              (F64, hx, None, 0)]), o, threads=THREADS)
    del ha, hb, hamt, hx
    want = o.export()
    del o
    assert got["keys"].shape[1] > 40_000_000
    assert_groups_equal(got, want, ["sum_d", "count", "min_f", "max_f"])


def test_highcard_2p28_resident_equals_8gb_cap_spill(ctx):
    n = 1 << 28
    resident, _ = _highcard(ctx, n, 1 << 26)
    spilled, peak = _highcard(ctx, n, 1 << 26, cap=8 << 30)
    assert peak <= 8 << 30
    assert resident["keys"].shape[1] > 65_000_000
    assert_groups_equal(resident, spilled, ["sum_d", "count", "min_f", "max_f"], rel=0.0)


def test_batched_512_queries_full_size(ctx):
    import wadjet_b200 as wg
    from wadjet_b200 import autotune, synth
    qs, keep = [], []
    for q in range(512):
        key, val, filt, card, thr = synth.batched_query(ctx, q)
        vt = I64 if q % 2 == 0 else F64
        qs.append({"batch": wg.Batch([wg.Column(I64, key), wg.Column(vt, val), wg.Column(I32, filt)]),
                   "group_by": [0], "aggs": [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1),
                                             wg.AggColumn(wg.AGG_MIN, 1), wg.AggColumn(wg.AGG_MAX, 1)],
                   "filters": [(2, wg.OP_LT, thr)], "ndv_hint": card})
        keep.append((key, val, filt, vt, thr))
    bq = wg.BatchedQueries(ctx, qs, autotune.load_tuned())
    counts = bq.run()
    for q, (key, val, filt, vt, thr) in enumerate(keep):
        got = bq.export(q, int(counts[q]))
        o = ob.Agg([0], [(0, 1, 0), (1, -1, 0), (2, 1, 0), (3, 1, 0)])
        ob.pipeline(ob.HostBatch([(I64, key.cpu().numpy(), None, 0), (vt, val.cpu().numpy(), None, 0),
                                  (I32, filt.cpu().numpy(), None, 0)]), o, filters=[(2, 2, thr)], threads=THREADS)
        k = ["sum_i", "count", "min_i", "max_i"] if vt == I64 else ["sum_f", "count", "min_f", "max_f"]
        assert_groups_equal(got, o.export(), k)
    bq.close()
