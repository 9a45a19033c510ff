"""Parquet pages decoded on the device (wg_batch_decode) against the oracle's CPU
decode and the source values, and the decoded batch feeding the fused pipeline.

- The reference's own RLE / bit-packed vectors (rle_test.go) decoded on the
  device as dictionary indices over an identity dictionary.
- PLAIN and dictionary pages of every column class, with and without NULL rows,
  over pages of uneven sizes (bit-exact, with the NULL rows' validity).
- Malformed pages (indices past the dictionary, levels that end early) fail
  with WG_E_INVALID and leave the context usable.
- wg_batch_upload: the decoded host batch uploaded as it is.
"""
import json
import os

import numpy as np
import pytest

from oracle import binding as ob
from tests.helpers import DEC_DTYPE, assert_groups_equal, dec_array

pytestmark = pytest.mark.gpu

I32, I64, F32, F64, DATE, DEC = 1, 2, 3, 4, 16, 17
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


class _DevBytes:
    """A device byte range torch can wrap (the CUDA array interface)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 2}


def _device_values(wg, b, col, dtype, n):
    """Column `col` of a device batch read back: (values, valid bool per row or None)."""
    import torch
    data, vw = b.column_pointer(col)
    torch.cuda.synchronize()
    nbytes = np.dtype(dtype).itemsize * n
    host = np.zeros(n, dtype)
    if n:
        host = torch.as_tensor(_DevBytes(data, nbytes), device="cuda").cpu().numpy().view(dtype)[:n]
    valid = None
    if vw:
        words = (n + 63) // 64
        raw = torch.as_tensor(_DevBytes(vw, words * 8), device="cuda").cpu().numpy()
        valid = np.unpackbits(raw, bitorder="little")[:n].astype(bool)
    return host, valid


@pytest.mark.parametrize("case", GOLD["rle"], ids=lambda c: c["ref"])
def test_reference_rle_vectors_on_the_device(ctx, case):
    import wadjet_b200 as wg
    from wadjet_b200 import pages
    bw, n = case["bit_width"], case["count"]
    ident = np.arange(max(1, 1 << bw), dtype=np.int32)
    ch = pages.Chunk(I32, [pages.Page(n, bytes([bw]) + bytes(case["data"]), pages.ENC_RLE_DICTIONARY)],
                     dictionary=ident)
    b = wg.DeviceBatch.decode(ctx, [ch])
    got, valid = _device_values(wg, b, 0, np.int32, n)
    assert valid is None
    assert got.tolist() == case["expect"]
    b.close()


@pytest.mark.parametrize("t,dtype", [(I32, np.int32), (I64, np.int64), (F32, np.float32), (F64, np.float64),
                                     (DATE, np.int32), (DEC, DEC_DTYPE)])
@pytest.mark.parametrize("nulls", [0.0, 0.1])
@pytest.mark.parametrize("dictionary", [False, True])
def test_chunks_match_oracle_and_source(ctx, t, dtype, nulls, dictionary):
    import wadjet_b200 as wg
    from wadjet_b200 import pages
    rng = np.random.default_rng(t * 10 + int(nulls * 10) + dictionary)
    n = 250_003
    card = 3000
    if t == DEC:
        vals = dec_array(rng.integers(-10**12, 10**12, card))[rng.integers(0, card, n)]
    elif t in (F32, F64):
        vals = (rng.standard_normal(card) * 1000).astype(dtype)[rng.integers(0, card, n)]
    else:
        vals = rng.integers(-10**6, 10**6, card).astype(dtype)[rng.integers(0, card, n)]
    valid = rng.random(n) >= nulls if nulls else None
    ch = pages.chunk(vals, t, valid, page_rows=77_777, dictionary=dictionary, scale=2 if t == DEC else 0)
    want, want_ok = ob.page_decode(ch.to_c(), n, dtype)
    b = wg.DeviceBatch.decode(ctx, [ch])
    got, got_ok = _device_values(wg, b, 0, dtype, n)
    if valid is None:
        assert got_ok is None and want_ok.all()
    else:
        np.testing.assert_array_equal(got_ok, valid)
        np.testing.assert_array_equal(want_ok, valid)
    np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
    keep = valid if valid is not None else np.ones(n, bool)
    np.testing.assert_array_equal(got[keep].view(np.uint8), np.ascontiguousarray(vals[keep]).view(np.uint8))
    b.close()


def test_malformed_pages_are_refused(ctx):
    import wadjet_b200 as wg
    from wadjet_b200 import pages
    rng = np.random.default_rng(4)
    vals = rng.integers(0, 100, 5000).astype(np.int64)
    ch = pages.chunk(vals, I64, None, dictionary=True)
    ch.dictionary = ch.dictionary[:50]  # indices past the dictionary's end
    with pytest.raises(wg.WadjetGPUError) as ei:
        wg.DeviceBatch.decode(ctx, [ch])
    assert ei.value.status == wg._abi.WG_E_INVALID
    valid = rng.random(5000) > 0.5
    ch = pages.chunk(vals, I64, valid)
    p = ch.pages[0]
    ch.pages[0] = pages.Page(p.num_values, p.data, p.encoding, p.def_levels[: len(p.def_levels) // 3])
    with pytest.raises(wg.WadjetGPUError) as ei:
        wg.DeviceBatch.decode(ctx, [ch])
    assert ei.value.status == wg._abi.WG_E_INVALID
    # the context still decodes and runs
    ok = pages.chunk(vals, I64, valid)
    b = wg.DeviceBatch.decode(ctx, [ok])
    got, got_ok = _device_values(wg, b, 0, np.int64, 5000)
    np.testing.assert_array_equal(got_ok, valid)
    np.testing.assert_array_equal(got[valid], vals[valid])
    b.close()


def test_decoded_star_join_feeds_the_pipeline(ctx):
    """The star join over fact columns decoded on the device from Parquet-encoded pages
    (fk PLAIN, qty dictionary, price DECIMAL as INT64 PLAIN, disc PLAIN) equals the
    oracle over the same rows."""
    import wadjet_b200 as wg
    from wadjet_b200 import pages
    n, nd = 1 << 20, 1 << 22
    fk, qty, price, disc = ob.gen_starjoin_fact(n, threads=4)
    key, grp = ob.gen_starjoin_dim(nd)
    price = price.view(DEC_DTYPE)
    chunks = [pages.chunk(fk, I32), pages.chunk(qty, I32, dictionary=True), pages.chunk(price, DEC, scale=2),
              pages.chunk(disc, F64)]
    b = wg.DeviceBatch.decode(ctx, chunks)
    join = wg.HashJoin(ctx, 0, 0, payload=[1], build_row_hint=nd)
    join.build([wg.Batch([wg.Column(I32, key), wg.Column(I32, grp)])])
    agg = wg.HashAggregate(ctx, [4], [wg.AggColumn(wg.AGG_SUM, 5), wg.AggColumn(wg.AGG_SUM, 2)], ndv_hint=1000)
    expr = wg.Expr(F64, [wg.Expr.col(2), wg.Expr.const_f(1.0), wg.Expr.col(3), "-", "*"])
    wg.run_pipeline(ctx, b, agg, filters=[(1, wg.OP_GT, 10)], join=join, exprs=[expr], device=True)
    agg.finalize()
    oj = ob.Join(nd)
    oj.append(I32, key)
    o = ob.Agg([4], [(0, 5, 0), (0, 2, 0)])
    ob.pipeline(ob.HostBatch([(I32, fk, None, 0), (I32, qty, None, 0), (DEC, price, None, 2), (F64, disc, None, 0)]),
                o, filters=[(1, wg.OP_GT, 10)], join=oj, probe_key=0,
                build=ob.HostBatch([(I32, key, None, 0), (I32, grp, None, 0)]), payload=[1],
                exprs=[ob.expr(F64, [("col", 2), ("cf", 1.0), ("col", 3), "-", "*"])], threads=4)
    assert_groups_equal(agg.export(), o.export(), ["sum_f", "sum_d"])
    agg.close()
    join.close()
    b.close()


def test_batch_upload_runs_like_host_input(ctx):
    import wadjet_b200 as wg
    rng = np.random.default_rng(8)
    n = 300_000
    k = rng.integers(0, 2000, n).astype(np.int64)
    v = rng.integers(-100, 100, n).astype(np.int64)
    valid = rng.random(n) > 0.1
    host = wg.Batch([wg.Column(I64, k), wg.Column(I64, v, valid)])
    b = wg.DeviceBatch.upload(ctx, host)
    used = ctx.ledger()["used"]
    assert used >= n * 16  # the uploaded columns are charged to the ledger
    aggs = [wg.AggColumn(wg.AGG_SUM, 1), wg.AggColumn(wg.AGG_COUNT, 1)]
    g1 = wg.HashAggregate(ctx, [0], aggs, ndv_hint=2000)
    wg.run_pipeline(ctx, b, g1, device=True)
    g1.finalize()
    g2 = wg.HashAggregate(ctx, [0], aggs, ndv_hint=2000)
    wg.run_pipeline(ctx, host, g2)
    g2.finalize()
    assert_groups_equal(g1.export(), g2.export(), ["sum_i", "count"])
    for g in (g1, g2):
        g.close()
    b.close()
    assert ctx.ledger()["used"] <= used - n * 16
