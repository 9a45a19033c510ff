"""Benchmark tables generated in HBM (include/wadjet_synth.h) as torch CUDA tensors.

- ``starjoin(n)``  : fact fk int32 Zipf(1.1) over 2^22 keys, qty int32 U[1,50],
  price DECIMAL(15,2) as Int128, disc float64 U[0,0.1); dim of 2^22 unique keys with grp U[0,1000).
- ``groupby(n)``   : k int64 U[0,4096), v int64 U[0,1e6), f float64 U[0,1), flag int32 U[0,10).
- ``highcard(n)``  : a int32, b int64 (~2^26 distinct (a,b)), amt DECIMAL(18,2), x float64 ~N(0,1).
- ``strgroup(n)``  : a BYTES column of n values drawn uniformly from `distinct` URL-like strings
  (8-56 lowercase bytes, the first five spelling the string's number in base 26, so all differ),
  as (offsets uint32, bytes uint8), and v int64 U[0,1e6).
"""
from __future__ import annotations

import torch

from . import _check, lib

SEED = 42
DIM_ROWS = 1 << 22


def _p(t):
    return t.data_ptr() if t is not None else None


def starjoin_fact(ctx, n: int, seed: int = SEED, row0: int = 0, device: int = 0):
    dev = torch.device("cuda", device)
    fk = torch.empty(n, dtype=torch.int32, device=dev)
    qty = torch.empty(n, dtype=torch.int32, device=dev)
    price = torch.empty((n, 2), dtype=torch.int64, device=dev)   # (hi, lo) per row
    disc = torch.empty(n, dtype=torch.float64, device=dev)
    _check(lib.wg_synth_starjoin_fact(ctx.h, seed, row0, n, _p(fk), _p(qty), _p(price), _p(disc)))
    return fk, qty, price, disc


def starjoin_dim(ctx, n: int = DIM_ROWS, seed: int = SEED, device: int = 0):
    dev = torch.device("cuda", device)
    key = torch.empty(n, dtype=torch.int32, device=dev)
    grp = torch.empty(n, dtype=torch.int32, device=dev)
    _check(lib.wg_synth_starjoin_dim(ctx.h, seed, n, _p(key), _p(grp)))
    return key, grp


def groupby(ctx, n: int, ngroups: int = 4096, seed: int = SEED, row0: int = 0, device: int = 0):
    dev = torch.device("cuda", device)
    k = torch.empty(n, dtype=torch.int64, device=dev)
    v = torch.empty(n, dtype=torch.int64, device=dev)
    f = torch.empty(n, dtype=torch.float64, device=dev)
    flag = torch.empty(n, dtype=torch.int32, device=dev)
    _check(lib.wg_synth_groupby(ctx.h, seed, row0, n, ngroups, _p(k), _p(v), _p(f), _p(flag)))
    return k, v, f, flag


def highcard(ctx, n: int, seed: int = SEED, row0: int = 0, device: int = 0):
    dev = torch.device("cuda", device)
    a = torch.empty(n, dtype=torch.int32, device=dev)
    b = torch.empty(n, dtype=torch.int64, device=dev)
    amt = torch.empty((n, 2), dtype=torch.int64, device=dev)
    x = torch.empty(n, dtype=torch.float64, device=dev)
    _check(lib.wg_synth_highcard(ctx.h, seed, row0, n, _p(a), _p(b), _p(amt), _p(x)))
    return a, b, amt, x


HC_KEY_SPACE = 1 << 26  # the b column's values are drawn uniformly from this many keys


def highcard_groups(n: int) -> int:
    """Expected distinct (a, b) groups among n rows of the high-cardinality table."""
    import math
    return int(HC_KEY_SPACE * -math.expm1(-n / HC_KEY_SPACE))


def batched_params(q: int, seed: int = SEED) -> tuple[int, int, int]:
    """(rows, key cardinality, filter threshold) of query q of the batched workload."""
    import ctypes as C
    r, c, t = C.c_int64(), C.c_int64(), C.c_int32()
    _check(lib.wg_synth_batched_params(seed, q, C.byref(r), C.byref(c), C.byref(t)))
    return r.value, c.value, t.value


def batched_query(ctx, q: int, seed: int = SEED, device: int = 0, rows: int | None = None):
    """Columns (key int64, value int64 for even q / float64 for odd q, filt int32) of query q."""
    n, card, thr = batched_params(q, seed)
    if rows is not None:
        n = rows
    dev = torch.device("cuda", device)
    key = torch.empty(n, dtype=torch.int64, device=dev)
    filt = torch.empty(n, dtype=torch.int32, device=dev)
    if q % 2 == 0:
        val = torch.empty(n, dtype=torch.int64, device=dev)
        _check(lib.wg_synth_batched(ctx.h, seed, q, n, card, _p(key), _p(val), None, _p(filt)))
    else:
        val = torch.empty(n, dtype=torch.float64, device=dev)
        _check(lib.wg_synth_batched(ctx.h, seed, q, n, card, _p(key), None, _p(val), _p(filt)))
    return key, val, filt, card, thr


def strgroup(n: int, distinct: int = 1 << 20, seed: int = SEED, device: int = 0, chunk: int = 1 << 22):
    """(offsets, bytes, v): see the module docstring. Generated with torch on the device."""
    dev = torch.device("cuda", device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    lens = torch.randint(8, 57, (distinct,), generator=g, device=dev, dtype=torch.int64)
    poff = torch.zeros(distinct + 1, dtype=torch.int64, device=dev)
    poff[1:] = torch.cumsum(lens, 0)
    pool = torch.randint(97, 123, (int(poff[-1]),), generator=g, device=dev, dtype=torch.int64).to(torch.uint8)
    ids = torch.arange(distinct, device=dev, dtype=torch.int64)
    for d in range(5):  # base-26 digits of the string's number
        pool[poff[:-1] + d] = (97 + (ids // (26 ** d)) % 26).to(torch.uint8)
    pick = torch.randint(0, distinct, (n,), generator=g, device=dev, dtype=torch.int64)
    plen = lens[pick]
    offs64 = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    offs64[1:] = torch.cumsum(plen, 0)
    total = int(offs64[-1])
    if total >= 1 << 32:
        raise ValueError("strgroup: more than 2^32 bytes")
    raw = torch.empty(total, dtype=torch.uint8, device=dev)
    for r0 in range(0, n, chunk):
        r1 = min(n, r0 + chunk)
        b0, b1 = int(offs64[r0]), int(offs64[r1])
        src = torch.repeat_interleave(poff[pick[r0:r1]] - offs64[r0:r1], plen[r0:r1]) + \
            torch.arange(b0, b1, device=dev, dtype=torch.int64)
        raw[b0:b1] = pool[src]
    v = torch.randint(0, 1_000_000, (n,), generator=g, device=dev, dtype=torch.int64)
    return offs64.to(torch.int32), raw, v
