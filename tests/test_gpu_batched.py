"""Batched mode (many queries in one persistent graph-replayed launch) against the
oracle run query by query: each query's groups must be what its own
Pipeline.Run produces."""
import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import assert_groups_equal

pytestmark = pytest.mark.gpu

I32, I64, F64, DEC = 1, 2, 4, 17


def make_queries(ctx, nq, max_rows, hint_scale=1.0):
    import wadjet_b200 as wg
    from wadjet_b200 import synth
    qs, host = [], []
    for q in range(nq):
        n, card, thr = synth.batched_params(q)
        n = min(n, max_rows)
        key, val, filt, card, thr = synth.batched_query(ctx, q, rows=n)
        vt = I64 if q % 2 == 0 else F64
        batch = wg.Batch([wg.Column(I64, key), wg.Column(vt, val), wg.Column(I32, filt)])
        aggs = [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_MIN, 1),
                wg.AggColumn(wg.AGG_MAX, 1)]
        qs.append({"batch": batch, "group_by": [0], "aggs": aggs, "filters": [(2, wg.OP_LT, thr)],
                   "ndv_hint": max(1, int(card * hint_scale)), "_keep": (key, val, filt)})
        host.append((key.cpu().numpy(), val.cpu().numpy(), filt.cpu().numpy(), vt, thr))
    return qs, host


def oracle_query(key, val, filt, vt, thr):
    o = ob.Agg([0], [(0, 1, 0), (1, -1, 0), (2, 1, 0), (3, 1, 0)])
    ob.pipeline(ob.HostBatch([(I64, key, None, 0), (vt, val, None, 0), (I32, filt, None, 0)]), o,
                filters=[(2, 2, thr)], threads=4)
    return o.export()


def kinds(vt):
    return ["sum_i", "count", "min_i", "max_i"] if vt == I64 else ["sum_f", "count", "min_f", "max_f"]


@pytest.mark.parametrize("params", [None, "nosmem", "small_tiles", "generic"])
def test_batched_matches_oracle(ctx, params, monkeypatch):
    import wadjet_b200 as wg
    # "generic": the kernel that reads the query shape at run time instead of the compiled shapes
    monkeypatch.setenv("WG_SPECIALIZE", "0" if params == "generic" else "1")
    tp = {None: None, "generic": None, "nosmem": wg.TuneParams(smem_max_groups=-1),
          "small_tiles": wg.TuneParams(tile_rows=4096, block=256, ctas_per_sm=4)}[params]
    qs, host = make_queries(ctx, 24, 300_000)
    b = wg.BatchedQueries(ctx, qs, tp)
    for _ in range(2):  # the graph is replayed: the second run must reset state
        counts = b.run()
    for q, (key, val, filt, vt, thr) in enumerate(host):
        want = oracle_query(key, val, filt, vt, thr)
        assert counts[q] == want["keys"].shape[1]
        assert_groups_equal(b.export(q, int(counts[q])), want, kinds(vt))
    b.close()


def test_batched_hint_too_small_is_rerun(ctx):
    """A query whose real group count overflows its hinted table is re-run on a
    grown table; results stay exact and the next replay uses the new table."""
    import wadjet_b200 as wg
    qs, host = make_queries(ctx, 6, 200_000, hint_scale=0.01)
    b = wg.BatchedQueries(ctx, qs, wg.TuneParams(max_load=0.75))
    for _ in range(2):
        counts = b.run()
        for q, (key, val, filt, vt, thr) in enumerate(host):
            want = oracle_query(key, val, filt, vt, thr)
            assert_groups_equal(b.export(q, int(counts[q])), want, kinds(vt))
    b.close()


def test_batched_queries_with_joins_match_oracle(ctx):
    """Batched queries that each run filter → hash-join probe → projection → GROUP BY in
    the one persistent launch (star-join shaped queries over fact slices of uneven sizes,
    sharing one resident dimension; plain group-by queries mixed in)."""
    import wadjet_b200 as wg
    from tests.helpers import DEC_DTYPE
    from wadjet_b200 import synth
    nd = 1 << 22
    key, grp = synth.starjoin_dim(ctx)
    join = wg.HashJoin(ctx, 0, 0, payload=[1], build_row_hint=nd)
    join.build([wg.Batch([wg.Column(I32, key), wg.Column(I32, grp)])], device=True)
    fk, qty, price, disc = synth.starjoin_fact(ctx, 3_000_000)
    expr = wg.Expr(F64, [wg.Expr.col(2), wg.Expr.const_f(1.0), wg.Expr.col(3), "-", "*"])
    qs, spans = [], []
    r0 = 0
    for q, n in enumerate([10_000, 250_000, 1_700_000, 40_000, 999_999]):
        b = wg.Batch([wg.Column(I32, fk[r0:r0 + n]), wg.Column(I32, qty[r0:r0 + n]),
                      wg.Column(DEC, price[r0:r0 + n], scale=2), wg.Column(F64, disc[r0:r0 + n])])
        qs.append({"batch": b, "group_by": [4], "aggs": [wg.AggColumn(wg.AGG_SUM, 5), wg.AggColumn(wg.AGG_SUM, 2),
                                                         wg.AggColumn(wg.AGG_COUNT, -1)],
                   "filters": [(1, wg.OP_GT, 10 + q)], "join": join, "exprs": [expr], "ndv_hint": 1000})
        spans.append((r0, n, 10 + q))
        r0 += n
    plain, host = make_queries(ctx, 3, 200_000)
    qs += plain
    bq = wg.BatchedQueries(ctx, qs)
    counts = bq.run()
    hkey, hgrp = key.cpu().numpy(), grp.cpu().numpy()
    oj = ob.Join(nd)
    oj.append(I32, hkey)
    hfk, hqty, hdisc = fk.cpu().numpy(), qty.cpu().numpy(), disc.cpu().numpy()
    hprice = price.cpu().numpy().reshape(-1).view(DEC_DTYPE)
    for q, (s0, n, thr) in enumerate(spans):
        o = ob.Agg([4], [(0, 5, 0), (0, 2, 0), (1, -1, 0)])
        ob.pipeline(ob.HostBatch([(I32, hfk[s0:s0 + n], None, 0), (I32, hqty[s0:s0 + n], None, 0),
                                  (DEC, hprice[s0:s0 + n], None, 2), (F64, hdisc[s0:s0 + n], None, 0)]), o,
                    filters=[(1, 4, thr)], join=oj, probe_key=0,
                    build=ob.HostBatch([(I32, hkey, None, 0), (I32, hgrp, None, 0)]), payload=[1],
                    exprs=[ob.expr(F64, [("col", 2), ("cf", 1.0), ("col", 3), "-", "*"])], threads=4)
        assert_groups_equal(bq.export(q, int(counts[q])), o.export(), ["sum_f", "sum_d", "count"])
    for i, h in enumerate(host):
        q = len(spans) + i
        assert_groups_equal(bq.export(q, int(counts[q])), oracle_query(*h), kinds(h[3]))
    bq.close()
    join.close()
