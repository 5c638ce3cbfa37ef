"""Several phenotype columns in one scan (the batched form): each trait with its own
missingness mask, so counts are mask-weighted; permuted copies of a trait (the reference's
-p rule, src/main.c:336-348). Every trait's per-pair counts, hits (trait-major order) and
maximum F are checked against the FP64 oracle run on that trait alone."""
import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu

F_TOL = 1e-5
TOL_SET = 1e-4


def _traits(nid, seed):
    rng = np.random.default_rng(seed)
    cols, valid = [], []
    base = rng.standard_normal(nid).astype(np.float32)
    for t in range(5):
        if t == 0:
            y = base
        elif t == 1:
            y = ((rng.gamma(2.0, 1.0, nid) - 2.0) / np.sqrt(2.0)).astype(np.float32)
        elif t == 2:
            y = (rng.standard_normal(nid) * 3.0 + 10.0).astype(np.float32)
        else:
            y = capi.permute_phenotype(base, t)  # permuted copies of trait 0
        cols.append(y)
        valid.append(rng.random(nid) >= [0.0, 0.05, 0.10, 0.02, 0.02][t])
    return np.stack(cols, 1), np.stack(valid, 1)


@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
@pytest.mark.parametrize("test", ["f", "i"])
def test_traits_each_match_oracle(gpu_ctx, form, test):
    nid, nsnp = 700, 160
    codes = synth.genotype_codes(nid, nsnp, seed=51)
    gp = synth.pack(codes)
    Y, V = _traits(nid, 52)
    T = Y.shape[1]
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    t2 = synth.f_threshold(4, nid - 9, 1e-2)
    blk = (0, nsnp, 0, nsnp)
    gpu_ctx.load_packed(gp, nid)
    gpu_ctx.set_traits(Y, V)
    opts = capi.default_opts(test=test, t1=t1, t2=t2, form=form, report_trait=-1)
    hits, total, ex = gpu_ctx.scan([blk], opts, ntraits=T, want_traits=True)
    assert np.all(np.diff(ex["trait"]) >= 0), "hits must be trait-major"
    tri = np.tril(np.ones((nsnp, nsnp), bool), -1)
    for t in range(T):
        phen = np.where(V[:, t], Y[:, t], np.float32(-9.0)).astype(np.float32)
        hb, tb, pb = oracles.oracle_scan_block(codes, phen, blk, test=test, t1=t1, t2=t2, per_pair=True)
        mine = hits[ex["trait"] == t]
        excl = parity.near_threshold(pb, blk, t1, t2, test, TOL_SET)
        ok, msg = parity.compare_hit_lists(mine, hb, excl)
        assert ok, "trait %d: %s" % (t, msg)
        if len(mine):
            assert parity.f_errors(mine, pb, blk, F_TOL).max() <= 1.0
        d = gpu_ctx.scan_dump(blk, capi.default_opts(test=test, t1=t1, t2=t2, form=form), trait=t)
        assert np.array_equal(d["counts"][tri], pb["counts"][tri]), "trait %d counts" % t
        fin = np.isfinite(pb["F"][tri])
        assert abs(ex["max_f"][t] - pb["F"][tri][fin].max()) <= F_TOL * max(1.0, pb["F"][tri][fin].max())


@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
def test_many_traits_global_maxima(gpu_ctx, form):
    """More traits than the kernels keep per-CTA maxima for in shared memory (512): the
    maxima fold into global memory directly. Every trait's largest F and F2 and a sample
    of traits' hit lists against the FP64 oracle."""
    nid, nsnp, T = 300, 48, 600
    codes = synth.genotype_codes(nid, nsnp, seed=61)
    gp = synth.pack(codes)
    rng = np.random.default_rng(62)
    base = rng.standard_normal(nid).astype(np.float32)
    Y = np.stack([base] + [capi.permute_phenotype(base, p) for p in range(1, T)], 1)
    V = rng.random((nid, T)) >= 0.02
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    t2 = synth.f_threshold(4, nid - 9, 1e-2)
    blk = (0, nsnp, 0, nsnp)
    gpu_ctx.load_packed(gp, nid)
    gpu_ctx.set_traits(Y, V)
    opts = capi.default_opts(test="i", t1=t1, t2=t2, form=form, report_trait=-1)
    hits, total, ex = gpu_ctx.scan([blk], opts, ntraits=T, want_traits=True)
    tri = np.tril(np.ones((nsnp, nsnp), bool), -1)
    for t in range(T):
        phen = np.where(V[:, t], Y[:, t], np.float32(-9.0)).astype(np.float32)
        hb, tb, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=t1, t2=t2, per_pair=True)
        for key, name in (("F", "max_f"), ("F2", "max_f2")):
            v = pb[key][tri]
            m = v[np.isfinite(v)].max()
            assert abs(ex[name][t] - m) <= F_TOL * max(1.0, m), "trait %d %s" % (t, key)
        if t in (0, 511, 512, 599):
            mine = hits[ex["trait"] == t]
            excl = parity.near_threshold(pb, blk, t1, t2, "i", TOL_SET)
            ok, msg = parity.compare_hit_lists(mine, hb, excl)
            assert ok, "trait %d: %s" % (t, msg)
