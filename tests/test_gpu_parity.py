"""GPU operators against the CPU oracle on the same seeded inputs (through the C ABI).

Integer, join and DECIMAL results must match bit for bit; float sums within
1e-12 relative (tests/helpers.py FLOAT_REL_TOL); float MIN/MAX exactly.
"""
import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import DEC_DTYPE, assert_groups_equal, dec_array, random_valid

pytestmark = pytest.mark.gpu

I32, I64, F32, F64, DATE, DEC = 1, 2, 3, 4, 16, 17


def rand_col(rng, t, n, lo=-1000, hi=1000):
    if t in (I32, DATE):
        return rng.integers(lo, hi, n, dtype=np.int32)
    if t == I64:
        return rng.integers(lo, hi, n, dtype=np.int64)
    if t == F32:
        return (rng.standard_normal(n) * 100).astype(np.float32)
    if t == F64:
        return rng.standard_normal(n) * 100
    return dec_array(rng.integers(-(10**12), 10**12, n))


# ---------------------------------------------------------------- filter --
@pytest.mark.parametrize("t", [I32, I64, F32, F64, DATE])
@pytest.mark.parametrize("n", [0, 1, 63, 4097, 100_003])
@pytest.mark.parametrize("nulls", [0.0, 0.1])
@pytest.mark.parametrize("use_sel", [False, True])
def test_filter_matches_oracle(ctx, t, n, nulls, use_sel):
    import wadjet_b200 as wg
    rng = np.random.default_rng(n * 7 + t)
    data = rand_col(rng, t, n)
    valid = random_valid(rng, n, nulls)
    sel = np.sort(rng.choice(n, size=n // 2, replace=False)).astype(np.uint32) if (use_sel and n) else None
    for op in range(6):
        const = 0.5 if t in (F32, F64) else 3
        want = ob.filter_(t, data, valid, op, const, sel=sel)
        f = wg.KernelFilter(ctx, 0, op, const)
        got = f.execute(wg.Batch([wg.Column(t, data, valid)], sel=sel))
        f.close()
        np.testing.assert_array_equal(got if got is not None else np.zeros(0, np.uint32), want)


def test_filter_device_unaligned_column(ctx):
    """A device column that starts off a 16-byte boundary takes the scalar path."""
    import torch
    import wadjet_b200 as wg
    rng = np.random.default_rng(5)
    host = rng.integers(0, 10, 10_001, dtype=np.int32)
    dev = torch.from_numpy(host).cuda()
    view = dev[1:]
    out = torch.empty(10_000, dtype=torch.int32, device="cuda")
    f = wg.KernelFilter(ctx, 0, wg.OP_LT, 7)
    n = f.execute_device(wg.Batch([wg.Column(I32, view)]), out)
    want = ob.filter_(I32, host[1:], None, wg.OP_LT, 7)
    np.testing.assert_array_equal(out[:n].cpu().numpy().view(np.uint32), want)
    f.close()


# ------------------------------------------------------------------ join --
@pytest.mark.parametrize("kt", [I32, I64])
@pytest.mark.parametrize("dups", [False, True])
@pytest.mark.parametrize("nulls", [0.0, 0.05])
def test_join_matches_oracle(ctx, kt, dups, nulls):
    import wadjet_b200 as wg
    rng = np.random.default_rng(11 + kt + 2 * dups)
    nb, npr = 20_000, 50_000
    dt = np.int32 if kt == I32 else np.int64
    bkeys = (rng.integers(0, 5_000 if dups else 1 << 30, nb) if dups else rng.permutation(1 << 20)[:nb]).astype(dt)
    if kt == I64:
        bkeys = bkeys * np.int64(0x100000001) - 7  # spans the full int64 range
    pkeys = bkeys[rng.integers(0, nb, npr)].copy()
    pkeys[::7] = (pkeys[::7] + 1)  # some misses
    bvalid = random_valid(rng, nb, nulls)
    pvalid = random_valid(rng, npr, nulls)
    sel = np.sort(rng.choice(npr, size=npr // 3, replace=False)).astype(np.uint32)
    j = wg.HashJoin(ctx, 0, 0, payload=[1])
    pay = np.arange(nb, dtype=np.int64)
    j.build([wg.Batch([wg.Column(kt, bkeys[: nb // 2], None if bvalid is None else bvalid[: nb // 2]),
                       wg.Column(I64, pay[: nb // 2])]),
             wg.Batch([wg.Column(kt, bkeys[nb // 2:], None if bvalid is None else bvalid[nb // 2:]),
                       wg.Column(I64, pay[nb // 2:])])])
    oj = ob.Join()
    oj.append(kt, bkeys, bvalid)
    assert j.stats()[1] == oj.distinct()
    for s in (None, sel):
        want = sorted(zip(*[a.tolist() for a in oj.probe(kt, pkeys, pvalid, sel=s)]))
        got = []
        for pr, br in j.probe(wg.Batch([wg.Column(kt, pkeys, pvalid)], sel=s), cap=7_777):
            got += list(zip(pr.tolist(), br.tolist()))
        assert sorted(got) == want
        # payload gather of the matched build rows
        if got:
            brows = np.array([b for _, b in got[:1000]], np.int64)
            vals, ok = j.gather(0, brows, np.int64)
            np.testing.assert_array_equal(vals, pay[brows])
            assert ok.all()
    j.close()


@pytest.mark.parametrize("dup", [False, True])
@pytest.mark.parametrize("probe_first", [False, True])
@pytest.mark.parametrize("full", [False, True])
def test_join_dense_unique_build(ctx, dup, probe_first, full):
    """Unique int32 keys over a narrow range with one int32 payload: the build makes only
    the dense direct table (payloads alone when the keys fill their range), and the hash
    index waits for the first non-fused probe. A duplicate key sends the build down the
    hash path. The fused pipeline (GROUP BY the payload), the pair probe, the payload
    gather and the build stats agree with the oracle whichever of the fused and non-fused
    calls comes first."""
    import wadjet_b200 as wg
    rng = np.random.default_rng(5 + dup)
    nb, npr = 30_000, 200_000
    bkeys = (rng.permutation(nb if full else 40_000)[:nb] + 1000).astype(np.int32)
    if dup:
        bkeys[-1] = bkeys[0]
    grp = rng.integers(0, 300, nb).astype(np.int32)
    pkeys = rng.integers(900, 41_100, npr).astype(np.int32)
    j = wg.HashJoin(ctx, 0, 0, payload=[1])
    j.build([wg.Batch([wg.Column(I32, bkeys), wg.Column(I32, grp)])])
    oj = ob.Join()
    oj.append(I32, bkeys, None)
    assert j.stats()[1] == oj.distinct()

    def fused():
        g = wg.HashAggregate(ctx, [1], [wg.AggColumn(wg.AGG_COUNT, -1)], ndv_hint=300)
        wg.run_pipeline(ctx, wg.Batch([wg.Column(I32, pkeys)]), g, join=j)
        g.finalize()
        o = ob.Agg([1], [(1, -1, 0)])
        ob.pipeline(ob.HostBatch([(I32, pkeys, None, 0)]), o, join=oj, probe_key=0,
                    build=ob.HostBatch([(I32, bkeys, None, 0), (I32, grp, None, 0)]), payload=[1], threads=8)
        assert_groups_equal(g.export(), o.export(), ["count"])
        g.close()

    def probe():
        want = sorted(zip(*[a.tolist() for a in oj.probe(I32, pkeys, None)]))
        got = []
        for pr, br in j.probe(wg.Batch([wg.Column(I32, pkeys)]), cap=50_000):
            got += list(zip(pr.tolist(), br.tolist()))
        assert sorted(got) == want
        brows = np.array([b for _, b in got[:1000]], np.int64)
        vals, ok = j.gather(0, brows, np.int32)
        np.testing.assert_array_equal(vals, grp[brows])
        assert ok.all()

    for step in ((probe, fused) if probe_first else (fused, probe)):
        step()
    j.close()


# ------------------------------------------------------------- aggregate --
AGG_KINDS = {  # (func, input type) -> comparison kind
    (0, I32): "sum_i", (0, I64): "sum_i", (0, F64): "sum_f", (0, F32): "sum_f", (0, DEC): "sum_d",
    (1, I64): "count", (1, None): "count",
    (2, I32): "min_i", (2, I64): "min_i", (2, F64): "min_f", (2, F32): "min_f", (2, DEC): "min_d",
    (3, I32): "max_i", (3, I64): "max_i", (3, F64): "max_f", (3, F32): "max_f", (3, DEC): "max_d",
    (4, I32): "avg_i", (4, I64): "avg_f", (4, F64): "avg_f", (4, DEC): "avg_d",
}


def agg_setup(rng, n, key_types, ncard, nulls, key_nulls):
    """Columns: keys..., then I32, I64, F32, F64, DEC value columns."""
    cols, ocols = [], []
    for kt in key_types:
        dt = np.int32 if kt == I32 else np.int64
        k = rng.integers(-ncard // 2, ncard // 2, n).astype(dt)
        if kt == I64:
            k = k * np.int64(0x9E3779B97F4A7C1) + 3
            k[k == np.int64(-0x7FFFFFFFFFFFFFFF)] = 0  # see test_int_hash_sentinel_key_is_one_group
        kv = random_valid(rng, n, key_nulls)
        cols.append((kt, k, kv))
    for t in (I32, I64, F32, F64, DEC):
        cols.append((t, rand_col(rng, t, n), random_valid(rng, n, nulls)))
    return cols


def make_aggs(nk):
    base = nk
    specs = [(0, base + 0), (0, base + 1), (0, base + 3), (0, base + 4), (1, -1), (1, base + 1),
             (2, base + 0), (3, base + 3), (2, base + 4), (3, base + 2), (4, base + 1)]
    types = {base + 0: I32, base + 1: I64, base + 2: F32, base + 3: F64, base + 4: DEC}
    kinds = [AGG_KINDS[(f, types.get(c) if c >= 0 else None)] for f, c in specs]
    return specs, kinds


def oracle_magnitude(cols, key_idx, specs):
    """The oracle's per-group sum(|x|) (mean(|x|) for AVG) of every float aggregate: the scale that the
    rounding error of a float sum taken in another order is proportional to."""
    acols, idx = list(cols), {}
    for i, (t, d, v) in enumerate(cols):
        if t in (F32, F64):
            idx[i] = len(acols)
            acols.append((t, np.abs(d), v))
    om = ob.Agg(key_idx, [(f, idx.get(c, c), 0) for f, c in specs])
    om.consume(ob.HostBatch([(t, d, v, 2 if t == DEC else 0) for t, d, v in acols]))
    return om.export()


def run_both(ctx, cols, key_idx, specs, hint=0, batches=3, device=False):
    import torch
    import wadjet_b200 as wg
    n = len(cols[0][1])
    bounds = np.linspace(0, n, batches + 1).astype(int)
    bounds = (bounds // 64) * 64
    bounds[-1] = n
    # the GPU and the oracle each take at most 8 aggregates per handle
    results = []
    for part in (specs[:6], specs[6:]):
        g = wg.HashAggregate(ctx, key_idx, [wg.AggColumn(f, c) for f, c in part], ndv_hint=hint)
        o = ob.Agg(key_idx, [(f, c, 0) for f, c in part])
        for a, b in zip(bounds[:-1], bounds[1:]):
            sl = [(t, d[a:b], None if v is None else v[a:b]) for t, d, v in cols]
            if device:
                gcols = []
                for t, d, v in sl:
                    td = torch.from_numpy(d.view(np.int64).reshape(-1, 2) if t == DEC else d).cuda()
                    vw = torch.from_numpy(wg.pack_validity(v).view(np.int64)).cuda() if v is not None else None
                    gcols.append(wg.Column(t, td, vw, 2 if t == DEC else 0))
                g.consume(wg.Batch(gcols), device=True)
            else:
                g.consume(wg.Batch([wg.Column(t, d, v, 2 if t == DEC else 0) for t, d, v in sl]))
            o.consume(ob.HostBatch([(t, d, v, 2 if t == DEC else 0) for t, d, v in sl]))
        g.finalize()
        results.append((g.export(), o.export(), g, o, oracle_magnitude(cols, key_idx, part)))
    return results


@pytest.mark.parametrize("key_types,ncard", [([I64], 5000), ([I32], 300), ([I32, I64], 20_000), ([], 1)])
@pytest.mark.parametrize("nulls,key_nulls", [(0.0, 0.0), (0.1, 0.05)])
def test_aggregate_matches_oracle(ctx, key_types, ncard, nulls, key_nulls):
    rng = np.random.default_rng(ncard + len(key_types))
    cols = agg_setup(rng, 60_000, key_types, ncard, nulls, key_nulls)
    specs, kinds = make_aggs(len(key_types))
    res = run_both(ctx, cols, list(range(len(key_types))), specs)
    assert_groups_equal(res[0][0], res[0][1], kinds[:6], magnitude=res[0][4])
    assert_groups_equal(res[1][0], res[1][1], kinds[6:], magnitude=res[1][4])
    for g in (res[0][2], res[1][2]):
        g.close()


def test_aggregate_device_batches_and_growth(ctx):
    """Device-resident batches, a hint far below the real group count (forces
    overflow replay and table growth), and the shared-memory path on a small hint."""
    rng = np.random.default_rng(3)
    cols = agg_setup(rng, 200_000, [I64], 150_000, 0.0, 0.0)
    specs, kinds = make_aggs(1)
    res = run_both(ctx, cols, [0], specs, hint=16, batches=4, device=True)
    assert_groups_equal(res[0][0], res[0][1], kinds[:6], magnitude=res[0][4])
    assert_groups_equal(res[1][0], res[1][1], kinds[6:], magnitude=res[1][4])


def test_large_table_growth_with_chunked_reservations(ctx):
    """2^23 rows of near-unique int64 keys into a table sized for 2^22 groups: the table is large
    enough that threads reserve groups several at a time, and it has to grow mid-run; every row
    must still land exactly once."""
    import torch
    import wadjet_b200 as wg
    rng = np.random.default_rng(23)
    n = 1 << 23
    k = (rng.integers(0, 1 << 40, n).astype(np.int64) * 3) + 1
    v = rng.integers(-1000, 1000, n).astype(np.int64)
    g = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_SUM, 1)], ndv_hint=1 << 22)
    wg.run_pipeline(ctx, wg.Batch([wg.Column(I64, torch.from_numpy(k).cuda()), wg.Column(I64, torch.from_numpy(v).cuda())]),
                    g, device=True)
    g.finalize()
    o = ob.Agg([0], [(1, -1, 0), (0, 1, 0)])
    ob.pipeline(ob.HostBatch([(I64, k, None, 0), (I64, v, None, 0)]), o, threads=8)
    assert_groups_equal(g.export(), o.export(), ["count", "sum_i"])
    g.close()


def test_aggregate_low_cardinality_smem(ctx):
    rng = np.random.default_rng(4)
    cols = agg_setup(rng, 300_000, [I64], 900, 0.0, 0.0)
    specs, kinds = make_aggs(1)
    res = run_both(ctx, cols, [0], specs, hint=1000, batches=2)
    assert_groups_equal(res[0][0], res[0][1], kinds[:6], magnitude=res[0][4])
    assert_groups_equal(res[1][0], res[1][1], kinds[6:], magnitude=res[1][4])


def test_clone_and_merge(ctx):
    """CloneSink per worker + MergeSink equals one serial aggregate (partitioned_agg_test.go:91)."""
    import wadjet_b200 as wg
    rng = np.random.default_rng(9)
    cols = agg_setup(rng, 80_000, [I64], 3000, 0.1, 0.02)
    specs, kinds = make_aggs(1)
    specs, kinds = specs[:6], kinds[:6]
    primary = wg.HashAggregate(ctx, [0], [wg.AggColumn(f, c) for f, c in specs])
    o = ob.Agg([0], [(f, c, 0) for f, c in specs])
    o.consume(ob.HostBatch([(t, d, v, 2 if t == DEC else 0) for t, d, v in cols]))
    workers = [primary.clone_sink() for _ in range(3)]
    for w, (a, b) in zip(workers, [(0, 25_600), (25_600, 51_200), (51_200, 80_000)]):
        w.consume(wg.Batch([wg.Column(t, d[a:b], None if v is None else v[a:b], 2 if t == DEC else 0)
                            for t, d, v in cols]))
    for w in workers:
        primary.merge_sink(w)
        w.close()
    primary.finalize()
    assert_groups_equal(primary.export(), o.export(), kinds, magnitude=oracle_magnitude(cols, [0], specs))
    primary.close()


def test_emit_pages_match_oracle(ctx):
    """Finalized output (writeAccToColumn) page by page against the oracle's emit."""
    import wadjet_b200 as wg
    rng = np.random.default_rng(10)
    cols = agg_setup(rng, 30_000, [I32], 5000, 0.1, 0.05)
    specs = [(0, 1), (0, 5), (1, -1), (2, 4), (4, 2)]
    g = wg.HashAggregate(ctx, [0], [wg.AggColumn(f, c) for f, c in specs])
    g.consume(wg.Batch([wg.Column(t, d, v, 2 if t == DEC else 0) for t, d, v in cols]))
    o = ob.Agg([0], [(f, c, 0) for f, c in specs])
    o.consume(ob.HostBatch([(t, d, v, 2 if t == DEC else 0) for t, d, v in cols]))
    g.finalize()
    pages = []
    while True:
        p = g.next()
        if p is None:
            break
        assert len(p[0][0]) <= wg.BATCH_SIZE
        pages.append(p)
    got = [(np.concatenate([p[i][0] for p in pages]), np.concatenate([p[i][1] for p in pages])) for i in range(6)]
    want = o.emit([np.int32, np.float64, np.float64, np.int64, np.float64, np.float64])
    key_g = np.where(got[0][1], got[0][0].astype(np.int64), np.iinfo(np.int64).min)
    key_w = np.where(want[0][1], want[0][0].astype(np.int64), np.iinfo(np.int64).min)
    og, ow = np.argsort(key_g, kind="stable"), np.argsort(key_w, kind="stable")
    np.testing.assert_array_equal(key_g[og], key_w[ow])
    for i in range(1, 6):
        np.testing.assert_array_equal(got[i][1][og], want[i][1][ow])
        m = want[i][1][ow]
        np.testing.assert_allclose(got[i][0][og][m], want[i][0][ow][m], rtol=1e-12, atol=0)
    g.close()


def test_int_hash_sentinel_key_is_one_group(ctx):
    """The key -0x7FFFFFFFFFFFFFFF is the reference intHashTable's empty marker
    (internal/engine/exec/int_hash.go:42): inserting it leaves the slot looking
    empty, so the reference (and the oracle, which restates it) gives every row
    with that key a group of its own. On the GPU every key value, including the
    table's own sentinel, is one real group; this test pins that divergence."""
    import wadjet_b200 as wg
    sentinel = np.int64(-0x7FFFFFFFFFFFFFFF)
    k = np.array([1, sentinel, 2, sentinel, sentinel, 1], np.int64)
    v = np.arange(6, dtype=np.int64)
    g = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_SUM, 1)])
    g.consume(wg.Batch([wg.Column(I64, k), wg.Column(I64, v)]))
    g.finalize()
    e = g.export()
    got = dict(zip(e["keys"][0].tolist(), zip(e["count"][0].tolist(), e["i64"][1].tolist())))
    assert got == {1: (2, 5), 2: (1, 2), int(sentinel): (3, 1 + 3 + 4)}
    o = ob.Agg([0], [(1, -1, 0)])
    o.consume(ob.HostBatch([(I64, k, None, 0)]))
    assert o.groups() == 2 + 3  # the reference's behaviour: one group per sentinel row
    g.close()


def test_scalar_aggregate_over_no_input(ctx):
    """COUNT over nothing is 0, SUM/MIN are NULL (aggregate.go:4270)."""
    import wadjet_b200 as wg
    g = wg.HashAggregate(ctx, [], [wg.AggColumn(wg.AGG_COUNT, -1), wg.AggColumn(wg.AGG_SUM, 0)])
    assert g.finalize() == 1
    page = g.next()
    assert page[0][0][0] == 0 and page[0][1][0]
    assert not page[1][1][0]
    g.close()


def test_ledger_refuses_over_budget():
    """A reservation beyond the HBM budget fails with ErrMemoryExceeded and reserves nothing."""
    import wadjet_b200 as wg
    with wg.Context(0, hbm_budget=64 << 20) as c:
        before = c.ledger()["used"]
        with pytest.raises(wg.MemoryExceeded):
            c.reserve(1 << 40)
        assert c.ledger()["used"] == before
        g = wg.HashAggregate(c, [0], [wg.AggColumn(wg.AGG_COUNT, -1)], ndv_hint=1 << 30)
        with pytest.raises(wg.MemoryExceeded):
            g.consume(wg.Batch([wg.Column(I64, np.arange(10, dtype=np.int64))]))
        g.close()


@pytest.mark.parametrize("key_types", [[I32, I64], [I32, I32, I32], [I32, I32]])
def test_nullable_composite_keys_match_oracle(ctx, key_types):
    """A NULL in any column of a composite key is that column's own value (the generic
    path the reference migrates to, aggregate.go:1822-1840): rows agreeing on every
    non-NULL column and on which columns are NULL form one group."""
    import wadjet_b200 as wg
    rng = np.random.default_rng(len(key_types) * 13)
    n = 80_000
    cols = []
    for t in key_types:
        v = rng.integers(0, 40, n).astype(np.int32 if t == I32 else np.int64)
        cols.append((t, v, rng.random(n) > 0.15))
    val = rng.integers(-10**6, 10**6, n).astype(np.int64)
    cols.append((I64, val, None))
    nk = len(key_types)
    aggs = [(0, nk, 0), (1, -1, 0), (2, nk, 0)]
    g = wg.HashAggregate(ctx, list(range(nk)), [wg.AggColumn(f, c, o) for f, c, o in aggs], ndv_hint=1000)
    for r0, r1 in ((0, n // 2), (n // 2, n)):
        g.consume(wg.Batch([wg.Column(t, d[r0:r1], None if v is None else v[r0:r1]) for t, d, v in cols]))
    g.finalize()
    o = ob.Agg(list(range(nk)), aggs)
    o.consume(ob.HostBatch([(t, d, v, 0) for t, d, v in cols]))
    got, want = g.export(), o.export()
    assert (want["key_valid"] == 0).any()
    assert_groups_equal(got, want, ["sum_i", "count", "min_i"])
    g.close()


def test_nullable_key_filling_128_bits_is_refused(ctx):
    """Two int64 key columns take all 128 bits of the packed key: no room for the NULL
    field, so a NULL there is refused rather than merged into another group."""
    import wadjet_b200 as wg
    a = np.arange(100, dtype=np.int64)
    g = wg.HashAggregate(ctx, [0, 1], [wg.AggColumn(wg.AGG_COUNT, -1)], ndv_hint=100)
    with pytest.raises(wg.WadjetGPUError) as ei:
        g.consume(wg.Batch([wg.Column(I64, a, a % 7 != 0), wg.Column(I64, a)]))
    assert ei.value.status == wg._abi.WG_E_UNSUPPORTED
    g.close()


@pytest.mark.parametrize("n_keys", [7, 900])
def test_shared_table_float_sums_across_the_fixed_point_range(ctx, n_keys):
    """Low-cardinality float SUMs accumulate in the shared table as exact fixed point
    for 2^-12 <= |x| < 2^30 and in float for the rest (zeros, tiny and huge values, both
    signs): every group's sum equals the oracle's within the reordered-sum bound."""
    import wadjet_b200 as wg
    rng = np.random.default_rng(n_keys)
    n = 400_000
    k = rng.integers(0, n_keys, n).astype(np.int64)
    mag = 10.0 ** rng.uniform(-9, 13, n)
    v = np.where(rng.random(n) < 0.5, -mag, mag)
    v[rng.random(n) < 0.05] = 0.0
    v[rng.random(n) < 0.01] = 2.0 ** 30          # the first value past the fixed range
    v[rng.random(n) < 0.01] = 2.0 ** -12         # the smallest value inside it
    g = wg.HashAggregate(ctx, [0], [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, -1)], ndv_hint=n_keys)
    wg.run_pipeline(ctx, wg.Batch([wg.Column(I64, k), wg.Column(F64, v)]), g)
    g.finalize()
    o = ob.Agg([0], [(0, 1, 0), (1, -1, 0)])
    o.consume(ob.HostBatch([(I64, k, None, 0), (F64, v, None, 0)]))
    m = ob.Agg([0], [(0, 1, 0), (1, -1, 0)])
    m.consume(ob.HostBatch([(I64, k, None, 0), (F64, np.abs(v), None, 0)]))
    assert_groups_equal(g.export(), o.export(), ["sum_f", "count"], magnitude=m.export())
    g.close()
