"""Device side of the multi-rank exchange, on one GPU.

Two shards are aggregated into two partial aggregates (as two ranks would),
their groups are hash-partitioned by owner on the device
(wg_agg_partition_state), each owner merges the rows routed to it
(wg_agg_merge_state), and the owners' groups together must equal one
aggregate over the whole table (partitioned_agg_test.go:91, parallel =
serial). Owners must be exactly what partitionFor gives over the route hash
(fibHash for one int key, packedHash for a packed key, routeNullHash for the
NULL key), computed independently in numpy.
"""
import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import DEC_DTYPE, assert_groups_equal, dec_array

pytestmark = pytest.mark.gpu

I32, I64, F64, DEC = 1, 2, 4, 17


def _owner_split(wg, parts_aggs, shape, n_parts):
    """Partition every partial's groups by owner and merge each owner's rows."""
    owners = [wg.HashAggregate(parts_aggs[0].ctx, *shape) for _ in range(n_parts)]
    for a in parts_aggs:
        rows, counts = a.partition_state(n_parts)
        assert sum(counts) == rows.shape[0]
        lay = a.state_layout()
        off = 0
        for p in range(n_parts):
            owners[p].merge_state(lay, rows[off:off + counts[p]])
            off += counts[p]
    out = []
    for o in owners:
        o.finalize()
        out.append(o.export())
        o.close()
    return out


def _concat(exps):
    r = {}
    for k in ("keys", "key_valid", "count", "i64", "f64", "dec", "has"):
        r[k] = np.concatenate([e[k] for e in exps], axis=1)
    return r


@pytest.mark.parametrize("n_parts", [2, 3, 8])
def test_starjoin_partials_partition_and_merge(ctx, n_parts):
    import wadjet_b200 as wg
    from wadjet_b200.exchange import partition_for, route_hash_int
    n, nd = 1 << 20, 1 << 22
    fk, qty, price, disc = ob.gen_starjoin_fact(n, threads=4)
    key, grp = ob.gen_starjoin_dim(nd)
    join = wg.HashJoin(ctx, 0, 0, payload=[1], build_row_hint=nd)
    join.build([wg.Batch([wg.Column(I32, key), wg.Column(I32, grp)])])
    expr = wg.Expr(F64, [wg.Expr.col(2), wg.Expr.const_f(1.0), wg.Expr.col(3), "-", "*"])
    aggs = [wg.AggColumn(wg.AGG_SUM, 5), wg.AggColumn(wg.AGG_SUM, 2), wg.AggColumn(wg.AGG_COUNT, -1)]
    shape = ([4], aggs, 1000)
    partials = []
    for r0, r1 in ((0, n // 3), (n // 3, n)):  # two uneven shards, as two ranks
        a = wg.HashAggregate(ctx, *shape[:2], ndv_hint=1000)
        wg.run_pipeline(ctx, wg.Batch([wg.Column(I32, fk[r0:r1]), wg.Column(I32, qty[r0:r1]),
                                       wg.Column(DEC, price[r0:r1], scale=2), wg.Column(F64, disc[r0:r1])]),
                        a, filters=[(1, wg.OP_GT, 10)], join=join, exprs=[expr])
        partials.append(a)
    owned = _owner_split(wg, partials, ([4], aggs), n_parts)
    for p, e in enumerate(owned):
        assert (partition_for(route_hash_int(e["keys"][0]), n_parts) == p).all()
    got = _concat(owned)
    oj = ob.Join(nd)
    oj.append(I32, key)
    o = ob.Agg([4], [(0, 5, 0), (0, 2, 0), (1, -1, 0)])
    ob.pipeline(ob.HostBatch([(I32, fk, None, 0), (I32, qty, None, 0), (DEC, price.view(DEC_DTYPE), None, 2),
                              (F64, disc, None, 0)]), o, filters=[(1, wg.OP_GT, 10)], join=oj, probe_key=0,
                build=ob.HostBatch([(I32, key, None, 0), (I32, grp, None, 0)]), payload=[1],
                exprs=[ob.expr(F64, [("col", 2), ("cf", 1.0), ("col", 3), "-", "*"])], threads=4)
    assert_groups_equal(got, o.export(), ["sum_f", "sum_d", "count"])
    for a in partials:
        a.close()
    join.close()


def test_packed_and_null_keys_route_like_partition_for(ctx):
    """Packed (a int32, b int64) keys route by packedHash, a packed key with a NULL column
    and a NULL single key by routeNullHash (routeHashPacked / routeHashInt64)."""
    import wadjet_b200 as wg
    from wadjet_b200.exchange import (ROUTE_NULL_HASH, pack_key_words, partition_for, route_hash_int,
                                      route_hash_packed)
    rng = np.random.default_rng(17)
    n = 200_000
    a_col = rng.integers(0, 1 << 10, n, dtype=np.int32)
    b_col = rng.integers(-(1 << 40), 1 << 40, n, dtype=np.int64)
    amt = dec_array(rng.integers(-10**9, 10**9, n))
    x = rng.standard_normal(n)
    aggs = [wg.AggColumn(wg.AGG_SUM, 2), wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_MIN, 3),
            wg.AggColumn(wg.AGG_MAX, 3)]
    a_valid = rng.random(n) > 0.02  # NULLs in one composite-key column
    partials = []
    for r0, r1 in ((0, n // 2), (n // 2, n)):
        p = wg.HashAggregate(ctx, [0, 1], aggs, ndv_hint=n)
        p.consume(wg.Batch([wg.Column(I32, a_col[r0:r1], a_valid[r0:r1]), wg.Column(I64, b_col[r0:r1]),
                            wg.Column(DEC, amt[r0:r1], scale=2), wg.Column(F64, x[r0:r1])]))
        partials.append(p)
    lay = partials[0].state_layout()
    owned = _owner_split(wg, partials, ([0, 1], aggs), 4)
    for p, e in enumerate(owned):
        lo, hi = pack_key_words(e["keys"], lay, e["key_valid"])
        full = e["key_valid"].all(axis=0)
        h = np.where(full, route_hash_packed(lo, hi), np.uint64(ROUTE_NULL_HASH))
        assert (partition_for(h, 4) == p).all()
    whole = wg.HashAggregate(ctx, [0, 1], aggs, ndv_hint=n)
    whole.consume(wg.Batch([wg.Column(I32, a_col, a_valid), wg.Column(I64, b_col), wg.Column(DEC, amt, scale=2),
                            wg.Column(F64, x)]))
    whole.finalize()
    assert_groups_equal(_concat(owned), whole.export(), ["sum_d", "count", "min_f", "max_f"])
    for p in partials + [whole]:
        p.close()

    # one nullable int key: the NULL group goes where routeNullHash sends it
    k = rng.integers(0, 5000, n).astype(np.int64)
    valid = rng.random(n) > 0.05
    v = rng.integers(-1000, 1000, n).astype(np.int64)
    one = [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1)]
    partials = []
    for r0, r1 in ((0, n // 2), (n // 2, n)):
        p = wg.HashAggregate(ctx, [0], one, ndv_hint=5000)
        p.consume(wg.Batch([wg.Column(I64, k[r0:r1], valid[r0:r1]), wg.Column(I64, v[r0:r1])]))
        partials.append(p)
    owned = _owner_split(wg, partials, ([0], one), 3)
    null_owner = int(partition_for(np.array([ROUTE_NULL_HASH], np.uint64), 3)[0])
    for p, e in enumerate(owned):
        kv = e["key_valid"][0].astype(bool)
        assert (partition_for(route_hash_int(e["keys"][0][kv]), 3) == p).all()
        assert (~kv).sum() == (1 if p == null_owner else 0)
    whole = wg.HashAggregate(ctx, [0], one, ndv_hint=5000)
    whole.consume(wg.Batch([wg.Column(I64, k, valid), wg.Column(I64, v)]))
    whole.finalize()
    assert_groups_equal(_concat(owned), whole.export(), ["sum_i", "count"])
    for p in partials + [whole]:
        p.close()
