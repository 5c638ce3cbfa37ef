"""Comparison helpers for the parity tests."""
import numpy as np

import oracles


def pair_key(h):
    return list(zip(h["snp1"].tolist(), h["snp2"].tolist()))


def near_threshold(b_per_pair, block, t1, t2, test, tol):
    """Pairs (global snp1, snp2) whose FP64 F (or F2) lies within relative `tol` of its
    threshold, plus pairs with df1 <= 0 (F is 0/0 in exact arithmetic; the reference's
    float32 gives NaN or inf there depending on rounding)."""
    s1, m1, s2, m2 = block
    F, F2, d1 = b_per_pair["F"], b_per_pair["F2"], b_per_pair["df1"]
    with np.errstate(invalid="ignore"):
        near = np.abs(F - t1) <= tol * abs(t1)
        if test == "i":
            near |= np.abs(F2 - t2) <= tol * abs(t2)
    near |= (d1 <= 0)
    gx, gy = np.nonzero(near)
    return set(zip((gx + s1).tolist(), (gy + s2).tolist()))


def compare_hit_lists(got, ref, excluded):
    """Same pairs in the same order once `excluded` pairs are dropped from both."""
    a = [k for k in pair_key(got) if k not in excluded]
    b = [k for k in pair_key(ref) if k not in excluded]
    if a == b:
        return True, ""
    sa, sb = set(a), set(b)
    msg = "only in got: %s; only in ref: %s" % (sorted(sa - sb)[:5], sorted(sb - sa)[:5])
    if sa == sb:
        first = next(i for i, (x, y) in enumerate(zip(a, b)) if x != y)
        msg = "same set, order differs at %d: %s vs %s" % (first, a[first], b[first])
    return False, msg


def kappa(F, df1, df2):
    """Amplification of relative errors in the within-cell sum of squares:
    SSY/SSW = 1 + F*df1/df2. It is ~1 at the configs' sizes; a pair whose cells hold
    almost every individual alone (tiny N) can reach thousands, and then FP32 sums --
    the reference's own arithmetic included -- cannot give F to 1e-5."""
    F = np.asarray(F, dtype=np.float64)
    return 1.0 + np.abs(F) * np.maximum(df1, 0) / np.maximum(df2, 1)


def f_excess(got, ref, df1, df2, tol):
    """Error of F against the FP64 oracle divided by its allowed bound
    tol * kappa * max(|F|, 1): relative for F >= 1 (every threshold region), absolute for
    F < 1 where a relative error has no meaning as F -> 0. <= 1 passes. NaN references
    (no valid individual, df1 <= 0) are skipped (returned as 0)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    ok = np.isfinite(ref) & (np.asarray(df1) > 0) & (np.asarray(df2) > 0)
    out = np.zeros(ref.shape)
    err = np.abs(got[ok] - ref[ok]) / np.maximum(np.abs(ref[ok]), 1.0)
    out[ok] = err / (tol * kappa(ref[ok], np.asarray(df1)[ok], np.asarray(df2)[ok]))
    return out


def f_errors(got, b_per_pair, block, tol, field="F"):
    """Error/bound ratios of the hits' F (or F2) against the FP64 oracle."""
    s1, _, s2, _ = block
    gx, gy = got["snp1"] - s1, got["snp2"] - s2
    return f_excess(got[field], b_per_pair[field][gx, gy], b_per_pair["df1"][gx, gy],
                    b_per_pair["df2"][gx, gy], tol)
