"""GROUP BY one STRING / BYTES column (consumeBatchStrGroup,
internal/engine/exec/aggregate.go:3038): the device dictionary against the
oracle's restatement of the reference's group numbering (oracle.binding
.StrGroupIndex), then the accumulators against the oracle's aggregation over
those group indexes.

The dictionary numbers strings by first appearance in row (selection) order,
as the reference's strHashTable does, so ids must match the oracle's group
indexes exactly; integer state bit for bit, float sums within 1e-12 relative.
"""
import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import assert_groups_equal

pytestmark = pytest.mark.gpu

I32, I64, F64, STRING, BYTES = 1, 2, 4, 5, 6


def rand_strings(rng, n, n_distinct, max_len=40, long_frac=0.02, empty=True):
    """n values drawn from n_distinct strings: mostly short, some several
    hundred bytes long, the empty string among them."""
    pool = []
    for i in range(n_distinct):
        ln = int(rng.integers(300, 700)) if rng.random() < long_frac else int(rng.integers(0 if empty else 1, max_len))
        pool.append(bytes(rng.integers(0, 256, ln, dtype=np.uint8)) + i.to_bytes(4, "little")[: 1 if ln else 0])
    if empty:
        pool[0] = b""
    pick = rng.integers(0, n_distinct, n)
    return [pool[p] for p in pick]


def str_column(values, valid, type_id=BYTES, device=False):
    import torch
    import wadjet_b200 as wg
    col = wg.Column.strings([v if (valid is None or valid[i]) else None for i, v in enumerate(values)], type_id)
    if valid is not None:
        col.valid = np.asarray(valid, bool)
    if device:
        offs, raw = col.data
        words = wg.pack_validity(col.valid) if col.valid is not None else None
        col = wg.Column(type_id, (torch.from_numpy(offs.view(np.int32)).cuda(),
                                  torch.from_numpy(raw if raw.size else np.zeros(1, np.uint8)).cuda()),
                        torch.from_numpy(words.view(np.int64)).cuda() if words is not None else None)
    return col


AGGS = [(1, -1), (0, 1), (2, 2), (3, 3), (4, 1), (0, 3)]   # COUNT(*), SUM i64, MIN i32, MAX f64, AVG i64, SUM f64
KINDS = ["count", "sum_i", "min_i", "max_f", "avg_f", "sum_f"]


def payload(rng, n):
    """Float sums (AVG of the int64 column, SUM of the float one) over non-negative
    values, so the order-dependent rounding stays within 1e-12 of the sum."""
    return [(I64, rng.integers(0, 10**9, n, dtype=np.int64), None),
            (I32, rng.integers(-1000, 1000, n, dtype=np.int32), None),
            (F64, rng.random(n) * 100, None)]


def run_case(ctx, batches, type_id=BYTES, device=False, hint=0):
    """batches: list of (values, valid, sel, payload cols). Returns (gpu export, oracle export,
    gpu aggregate, oracle index)."""
    import wadjet_b200 as wg
    g = wg.HashAggregate(ctx, [0], [wg.AggColumn(f, c) for f, c in AGGS], ndv_hint=hint)
    o = ob.Agg([0], [(f, c, 0) for f, c in AGGS])
    idx = ob.StrGroupIndex()
    for values, valid, sel, pay in batches:
        cols = [str_column(values, valid, type_id, device)]
        for t, d, v in pay:
            if device:
                import torch
                cols.append(wg.Column(t, torch.from_numpy(d).cuda()))
            else:
                cols.append(wg.Column(t, d, v))
        dsel = sel
        if device and sel is not None:
            import torch
            dsel = torch.from_numpy(np.asarray(sel, np.uint32).view(np.int32)).cuda()
        g.consume(wg.Batch(cols, sel=dsel, length=len(values)), device=device)
        ids, ok = idx.map(values, valid, sel)
        o.consume(ob.HostBatch([(I32, ids, ok, 0)] + [(t, d, v, 0) for t, d, v in pay], sel=sel))
    g.finalize()
    return g.export(), o.export(), g, idx


def check(ctx, got, want, g, idx):
    assert_groups_equal(got, want, KINDS)
    ok = got["key_valid"][0].astype(bool)
    ids = got["keys"][0][ok]
    strs = idx.strings
    assert sorted(ids.tolist()) == list(range(len(strs)))
    assert g.key_strings(ids) == [strs[i] for i in ids]


@pytest.mark.parametrize("nulls", [0.0, 0.07])
def test_host_batches_match_oracle(ctx, nulls):
    rng = np.random.default_rng(11)
    batches = []
    for b in range(3):
        n = [20_000, 1, 35_001][b]
        vals = rand_strings(rng, n, 3000)
        valid = (rng.random(n) >= nulls) if nulls else None
        sel = np.sort(rng.choice(n, n // 2, replace=False)).astype(np.uint32) if b == 2 else None
        batches.append((vals, valid, sel, payload(rng, n)))
    got, want, g, idx = run_case(ctx, batches)
    check(ctx, got, want, g, idx)
    g.close()


def test_device_batches_grow_the_dictionary(ctx):
    """Device-resident string columns over two batches: about 110 000 distinct
    strings, then about 43 000 new ones added to the same dictionary."""
    rng = np.random.default_rng(12)
    batches = []
    for n, nd in [(200_000, 150_000), (50_000, 160_000)]:
        vals = rand_strings(rng, n, nd, max_len=24, long_frac=0.001)
        batches.append((vals, rng.random(n) >= 0.02, None, payload(rng, n)))
    got, want, g, idx = run_case(ctx, batches, device=True)
    check(ctx, got, want, g, idx)
    g.close()


def test_device_selection_and_string_type(ctx):
    rng = np.random.default_rng(13)
    n = 40_000
    vals = [s.decode("latin-1").encode() for s in rand_strings(rng, n, 500)]
    sel = np.sort(rng.choice(n, 9_000, replace=False)).astype(np.uint32)
    got, want, g, idx = run_case(ctx, [(vals, None, sel, payload(rng, n))], type_id=STRING, device=True)
    check(ctx, got, want, g, idx)
    g.close()


def test_emit_returns_strings(ctx):
    """Next() pages carry the key column as strings (None for the NULL key)."""
    import wadjet_b200 as wg
    vals = ["a", "bb", None, "", "a", "ccc", None, "bb", "é"]
    v = np.array([1, 2, 3, 4, 5, 6, 7, 8, 9], np.int64)
    g = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1)])
    g.consume(wg.Batch([wg.Column.strings(vals), wg.Column(I64, v)]))
    rows = g.collect()
    keys, kv = rows[0]
    got = {(keys[i] if kv[i] else None): (int(rows[1][0][i]), int(rows[2][0][i])) for i in range(len(keys))}
    assert got == {"a": (6, 2), "bb": (10, 2), None: (10, 2), "": (4, 1), "ccc": (6, 1), "é": (9, 1)}
    g.close()


def test_reset_numbers_from_zero_and_refusals(ctx):
    import wadjet_b200 as wg
    g = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_COUNT, -1)])
    g.consume(wg.Batch([wg.Column.strings(["x", "y", "x"])]))
    g.finalize()
    e = g.export()
    assert sorted(e["keys"][0].tolist()) == [0, 1] and g.key_strings([0, 1]) == [b"x", b"y"]
    # a string-keyed aggregate is not merged (two dictionaries number strings apart)
    other = g.clone_sink()
    other.consume(wg.Batch([wg.Column.strings(["z"])]))
    with pytest.raises(wg.WadjetGPUError):
        g.merge_sink(other)
    other.close()
    with pytest.raises(wg.WadjetGPUError):
        g.key_strings([2])
    g.reset()
    g.consume(wg.Batch([wg.Column.strings(["q", "x"])]))
    g.finalize()
    assert g.key_strings([0, 1]) == [b"q", b"x"]
    # an integer batch into a string-keyed aggregate is refused
    g.reset()
    with pytest.raises(wg.WadjetGPUError):
        g.consume(wg.Batch([wg.Column(I64, np.arange(4, dtype=np.int64))]))
    g.close()
    # a string column in a composite key is refused; so is key_strings on an int key
    c = wg.HashAggregate(ctx, [0, 1], [wg.AggColumn(wg.AGG_COUNT, -1)])
    with pytest.raises(wg.WadjetGPUError):
        c.consume(wg.Batch([wg.Column.strings(["a"]), wg.Column(I64, np.zeros(1, np.int64))]))
    c.close()
    h = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_COUNT, -1)])
    h.consume(wg.Batch([wg.Column(I64, np.arange(4, dtype=np.int64))]))
    h.finalize()
    with pytest.raises(wg.WadjetGPUError):
        h.key_strings([0])
    h.close()


def test_many_rows_properties(ctx):
    """4M rows over 1M distinct strings: every row counted once, one group per
    distinct string, and every id's string is the one its rows carried."""
    import torch
    import wadjet_b200 as wg
    rng = np.random.default_rng(14)
    n, nd = 1 << 22, 1 << 20
    lens = rng.integers(4, 28, nd)
    pool_offs = np.zeros(nd + 1, np.int64)
    pool_offs[1:] = np.cumsum(lens)
    pool = rng.integers(97, 123, int(pool_offs[-1]), dtype=np.uint8)
    pool[pool_offs[:-1]] = (np.arange(nd) % 26 + 65).astype(np.uint8)
    pick = rng.integers(0, nd, n)
    plens = lens[pick]
    offs = np.zeros(n + 1, np.int64)
    offs[1:] = np.cumsum(plens)
    starts = pool_offs[pick]
    gather = (np.repeat(starts - offs[:-1], plens) + np.arange(int(offs[-1]))).astype(np.int64)
    raw = pool[gather]
    col = wg.Column(BYTES, (torch.from_numpy(offs.astype(np.uint32).view(np.int32)).cuda(), torch.from_numpy(raw).cuda()))
    g = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_MIN, 1)])
    rows = torch.arange(n, dtype=torch.int64, device="cuda")
    g.consume(wg.Batch([col, wg.Column(I64, rows)]), device=True)
    ng = g.finalize()
    e = g.export()
    # distinct strings drawn (the pool's strings may repeat by chance)
    want_distinct = len({bytes(pool[pool_offs[p]:pool_offs[p + 1]]) for p in np.unique(pick)})
    assert ng == want_distinct
    assert int(e["count"][0].sum()) == n
    # each group's first row (MIN of the row number) holds the group's string,
    # and ids follow first appearance: sorting groups by first row sorts ids
    first = e["i64"][1]
    order = np.argsort(first)
    assert np.array_equal(e["keys"][0][order], np.arange(ng))
    sample = order[:: max(1, ng // 2000)]
    strs = g.key_strings(e["keys"][0][sample])
    for s, r in zip(strs, first[sample]):
        assert s == raw[offs[r]:offs[r + 1]].tobytes()
    g.close()


def by_string(export, strings_of, agg_cols):
    """{string or None: (count of agg 0, i64 of each agg in agg_cols)} from an export whose key holds ids."""
    out = {}
    ok = export["key_valid"][0].astype(bool)
    ids = export["keys"][0]
    names = strings_of(ids[ok]) if ok.any() else []
    it = iter(names)
    for g in range(export["count"].shape[1]):
        k = next(it) if ok[g] else None
        out[k] = (int(export["count"][0, g]),) + tuple(int(export["i64"][a, g]) for a in agg_cols)
    return out


@pytest.mark.parametrize("device", [False, True])
def test_pipeline_filter_and_join_with_string_key(ctx, device):
    """A fused filter -> hash probe -> aggregate whose GROUP BY column is a string of
    the probe side, against the oracle pipeline over the oracle's string numbering
    (compared by string: rows the filter or the join drop leave their strings in
    the device dictionary without a group, so ids may differ)."""
    import torch
    import wadjet_b200 as wg
    rng = np.random.default_rng(21)
    n = 60_000
    vals = rand_strings(rng, n, 2000, max_len=30)
    valid = rng.random(n) >= 0.03
    fk = rng.integers(0, 4000, n, dtype=np.int32)
    flag = rng.integers(0, 10, n, dtype=np.int32)
    v = rng.integers(0, 10**6, n, dtype=np.int64)
    bkeys = np.unique(rng.integers(0, 4000, 1500, dtype=np.int32))
    bgrp = rng.integers(0, 100, len(bkeys), dtype=np.int32)
    specs = [(1, -1), (0, 3)]   # COUNT(*), SUM(v)
    for use_join in (False, True):
        g = wg.HashAggregate(ctx, [0], [wg.AggColumn(f, c) for f, c in specs])
        j = None
        if use_join:
            j = wg.HashJoin(ctx, 0, 1, payload=[1])
            j.build([wg.Batch([wg.Column(I32, bkeys), wg.Column(I32, bgrp)])])
        sc = str_column(vals, valid, BYTES, device)
        cols = [sc] + [wg.Column(t, torch.from_numpy(d).cuda() if device else d)
                       for t, d in ((I32, fk), (I32, flag), (I64, v))]
        wg.run_pipeline(ctx, wg.Batch(cols), g, filters=[(2, wg.OP_LT, 6)], join=j, device=device)
        g.finalize()
        got = by_string(g.export(), g.key_strings, [1])
        # oracle: the strings numbered over all rows, then the oracle pipeline over the ids
        idx = ob.StrGroupIndex()
        ids, ok = idx.map(vals, valid)
        o = ob.Agg([0], [(f, c, 0) for f, c in specs])
        hb = ob.HostBatch([(I32, ids, ok, 0), (I32, fk, None, 0), (I32, flag, None, 0), (I64, v, None, 0)])
        if use_join:
            oj = ob.Join(len(bkeys))
            oj.append(I32, bkeys)
            ob.pipeline(hb, o, filters=[(2, wg.OP_LT, 6)], join=oj, probe_key=1,
                        build=ob.HostBatch([(I32, bkeys, None, 0), (I32, bgrp, None, 0)]), payload=[1])
        else:
            ob.pipeline(hb, o, filters=[(2, wg.OP_LT, 6)])
        strs = idx.strings
        want = by_string(o.export(), lambda x: [strs[i] for i in x], [1])
        assert got == want
        g.close()
        if j is not None:
            j.close()
