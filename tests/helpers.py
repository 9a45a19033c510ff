"""Shared test helpers: canonical-sort comparison of grouped results (the
reference's oracle compares result multisets after canonicalisation,
internal/oracle/compare.go) and small data builders."""
from __future__ import annotations

import numpy as np

FLOAT_REL_TOL = 1e-12  # float SUM: only the summation order differs from the reference


def canonical_order(exp: dict) -> np.ndarray:
    """Row order that sorts groups by (key_valid, key) over every key column."""
    keys, kv = exp["keys"], exp["key_valid"]
    if keys.shape[0] == 0:
        return np.arange(exp["count"].shape[1] if exp["count"].size else 0)
    cols = []
    for k in range(keys.shape[0] - 1, -1, -1):
        cols.append(keys[k])
        cols.append(kv[k])
    return np.lexsort(cols)


def assert_groups_equal(got: dict, want: dict, kinds: list[str], rel: float = FLOAT_REL_TOL,
                        magnitude: dict | None = None) -> None:
    """Compare two exported group tables after canonical sort.

    kinds[a] in {"count", "sum_i", "sum_f", "sum_d", "min_i", "max_i", "min_f", "max_f", "min_d", "max_d",
    "avg_i", "avg_f", "avg_d"}: integer / DECIMAL state must match bit for bit, float MIN/MAX exactly, and
    float sums within `rel` of their magnitude. A float sum taken in another order differs by rounding
    error proportional to sum(|x|), not to |sum(x)|, so when the inputs have mixed signs the caller
    passes `magnitude`: an export over the same groups whose float aggregate a holds sum(|x|) (mean(|x|)
    for AVG), and the bound becomes rel * max(|want|, magnitude).
    """
    ng, nw = got["count"].shape[1] if got["count"].size else got["keys"].shape[1], \
        want["count"].shape[1] if want["count"].size else want["keys"].shape[1]
    assert ng == nw, f"group count {ng} != {nw}"
    og, ow = canonical_order(got), canonical_order(want)
    om = canonical_order(magnitude) if magnitude is not None else None
    np.testing.assert_array_equal(got["key_valid"][:, og], want["key_valid"][:, ow])
    kvalid = want["key_valid"][:, ow].astype(bool)
    np.testing.assert_array_equal(np.where(kvalid, got["keys"][:, og], 0), np.where(kvalid, want["keys"][:, ow], 0))
    for a, kind in enumerate(kinds):
        cg, cw = got["count"][a, og], want["count"][a, ow]
        np.testing.assert_array_equal(cg, cw, err_msg=f"agg {a} count")
        has = want["has"][a, ow].astype(bool)
        np.testing.assert_array_equal(got["has"][a, og].astype(bool), has, err_msg=f"agg {a} has")
        if kind in ("sum_i", "min_i", "max_i", "avg_i"):
            np.testing.assert_array_equal(got["i64"][a, og][has], want["i64"][a, ow][has], err_msg=f"agg {a} i64")
        elif kind in ("sum_d", "min_d", "max_d", "avg_d"):
            np.testing.assert_array_equal(got["dec"][a, og][has], want["dec"][a, ow][has], err_msg=f"agg {a} dec")
        elif kind in ("sum_f", "avg_f"):
            g, w = got["f64"][a, og][has], want["f64"][a, ow][has]
            scale = np.abs(w)
            if magnitude is not None:
                scale = np.maximum(scale, np.abs(magnitude["f64"][a, om][has]))
            bad = ~(np.abs(g - w) <= rel * scale)
            assert not bad.any(), (f"agg {a} f64 sum: {int(bad.sum())} of {bad.size} groups differ by more than "
                                   f"{rel} of their magnitude; got {g[bad][:3]} want {w[bad][:3]}")
        elif kind in ("min_f", "max_f"):
            np.testing.assert_array_equal(got["f64"][a, og][has], want["f64"][a, ow][has], err_msg=f"agg {a} f64")


def random_valid(rng: np.random.Generator, n: int, null_frac: float):
    if null_frac <= 0:
        return None
    return rng.random(n) >= null_frac


DEC_DTYPE = np.dtype([("hi", "<i8"), ("lo", "<u8")])


def dec_array(vals) -> np.ndarray:
    """Int128 (hi, lo) array from Python ints (two's complement)."""
    out = np.zeros(len(vals), DEC_DTYPE)
    for i, v in enumerate(vals):
        v = int(v)
        out[i]["hi"] = -1 if v < 0 else 0
        out[i]["lo"] = v & (2**64 - 1)
    return out
