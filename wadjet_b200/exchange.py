"""Partial-aggregate exchange between ranks (one process per GPU).

Each rank aggregates its own shard of the fact table; the per-group partial
states are then combined the way MergeSink combines worker clones
(exec/aggregate.go:4682 → kernel.Accumulator.Merge, exec/kernel/types.go:106):
counts and sums add (int64 wrapping, Int128 exact, float64 in rank order), MIN
and MAX keep the extreme of the groups that have one. The states are tiny next
to the fact rows (one row per group), so they travel with one all-gather.
"""
from __future__ import annotations

import numpy as np

DEC_DTYPE = np.dtype([("hi", "<i8"), ("lo", "<u8")])
_M128 = (1 << 128) - 1


def shard_range(n_total: int, rank: int, world: int, align: int = 64) -> tuple[int, int]:
    """Rows [row0, row0 + n) of an n_total-row table owned by `rank` (aligned cuts)."""
    per = (n_total // world // align) * align
    row0 = rank * per
    n = n_total - row0 if rank == world - 1 else per
    return row0, n


def _dec_to_int(d: np.ndarray) -> list[int]:
    return [((int(h) << 64) | int(l)) if h >= 0 else ((int(h) << 64) | int(l)) for h, l in zip(d["hi"], d["lo"])]


def _int_to_dec(vals: list[int]) -> np.ndarray:
    out = np.zeros(len(vals), DEC_DTYPE)
    for i, v in enumerate(vals):
        v &= _M128
        hi = v >> 64
        out[i]["hi"] = hi - (1 << 64) if hi >= (1 << 63) else hi
        out[i]["lo"] = v & ((1 << 64) - 1)
    return out


def merge_exports(parts: list[dict], kinds: list[str]) -> dict:
    """Combine exported group tables (HashAggregate.export() layout) of several ranks.

    kinds[a] names aggregate a's state: count | sum_i | sum_f | sum_d | min_i | max_i | min_f | max_f |
    min_d | max_d | avg_i | avg_f | avg_d.
    """
    nk = parts[0]["keys"].shape[0]
    na = len(kinds)
    keys = np.concatenate([p["keys"] for p in parts], axis=1)
    kv = np.concatenate([p["key_valid"] for p in parts], axis=1)
    n = keys.shape[1]
    if nk:
        ident = np.stack([kv[k] for k in range(nk)] + [np.where(kv[k] != 0, keys[k], 0) for k in range(nk)], axis=1)
        uniq, inv = np.unique(ident, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        g = uniq.shape[0]
        out_kv = uniq[:, :nk].T.astype(np.uint8)
        out_keys = uniq[:, nk:].T.astype(np.int64)
    else:
        g, inv = (1 if n else 0), np.zeros(n, np.int64)
        out_kv = np.zeros((0, g), np.uint8)
        out_keys = np.zeros((0, g), np.int64)
    cat = {f: np.concatenate([p[f] for p in parts], axis=1) for f in ("count", "i64", "f64", "dec", "has")}
    r = {"keys": out_keys, "key_valid": out_kv, "count": np.zeros((na, g), np.int64),
         "i64": np.zeros((na, g), np.int64), "f64": np.zeros((na, g), np.float64),
         "dec": np.zeros((na, g), DEC_DTYPE), "has": np.zeros((na, g), np.uint8)}
    for a, kind in enumerate(kinds):
        np.add.at(r["count"][a], inv, cat["count"][a])
        has = cat["has"][a].astype(bool)
        hg = np.zeros(g, bool)
        np.logical_or.at(hg, inv, has)
        r["has"][a] = hg if kind.startswith(("min", "max")) else (r["count"][a] > 0)
        if kind in ("sum_i", "avg_i"):
            with np.errstate(over="ignore"):
                np.add.at(r["i64"][a], inv, cat["i64"][a])
        elif kind in ("sum_f", "avg_f"):
            np.add.at(r["f64"][a], inv, cat["f64"][a])
        elif kind in ("sum_d", "avg_d"):
            acc = [0] * g
            for i, v in zip(inv.tolist(), _dec_to_int(cat["dec"][a])):
                acc[i] += v
            r["dec"][a] = _int_to_dec(acc)
        elif kind in ("min_i", "max_i", "min_f", "max_f"):
            f = "i64" if kind.endswith("_i") else "f64"
            lo = kind.startswith("min")
            fill = (np.iinfo(np.int64).max if lo else np.iinfo(np.int64).min) if f == "i64" else (np.inf if lo else -np.inf)
            acc = np.full(g, fill, dtype=r[f].dtype)
            vals = np.where(has, cat[f][a], fill)
            (np.minimum if lo else np.maximum).at(acc, inv, vals)
            r[f][a] = np.where(hg, acc, 0)
        elif kind in ("min_d", "max_d"):
            best: list = [None] * g
            for i, v, h in zip(inv.tolist(), _dec_to_int(cat["dec"][a]), has.tolist()):
                if not h:
                    continue
                s = v - (1 << 128) if v >= (1 << 127) else v
                if best[i] is None or (s < best[i] if kind == "min_d" else s > best[i]):
                    best[i] = s
            r["dec"][a] = _int_to_dec([0 if b is None else b for b in best])
    return r
