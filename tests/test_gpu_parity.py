"""GPU parity: the CUDA scan forms against oracle A (the reference's own kernels run as
C) and oracle B (FP64 restatement), on seeded inputs small enough for the oracles.

Bars: cell counts and df bit-exact; the set and order of hits identical except pairs
whose FP64 F is within TOL_SET of a threshold (and df1 == 0 pairs, where the reference's
float32 gives NaN or inf by rounding); F and F2 within F_TOL * kappa * max(|F|, 1) of FP64
(relative for F >= 1, absolute below), kappa = SSY/SSW = 1 + F*df1/df2 (about 1 at the
configs' sizes, see parity.kappa).
"""
import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu

F_TOL = 1e-5      # F / F2 relative error against the FP64 oracle
TOL_SET = 1e-4    # threshold neighbourhood excluded from the hit-set comparison
FORMS = [capi.FORM_POPC, capi.FORM_TENSOR]
FORM_IDS = ["popc", "tensor"]


def _data(nid, nsnp, seed, miss_g=0.01, miss_p=0.02):
    codes = synth.genotype_codes(nid, nsnp, seed=seed, miss=miss_g)
    gp = synth.pack(codes)
    phen = synth.phenotype(nid, seed=seed + 1, miss=miss_p)
    return codes, gp, phen


def _check_block(ctx, codes, gp, phen, block, test, safe, t1, t2, form, chunk=128, check_ref=True):
    nid = codes.shape[1]
    ctx.load_packed(gp, nid)
    ctx.set_phenotype(phen, safe=safe)
    opts = capi.default_opts(test=test, safe=safe, chunk=chunk, t1=t1, t2=t2, form=form)
    got, total, ex = ctx.scan([block], opts, cap=1 << 22)
    assert total == len(got)
    hb, tb, pb = oracles.oracle_scan_block(codes, phen, block, test=test, safe=safe, chunk=chunk, t1=t1, t2=t2,
                                           per_pair=True)
    # per-pair dump: counts and df bit-exact against B, F against B
    d = ctx.scan_dump(block, opts)
    s1, m1, s2, m2 = block
    tri = (np.arange(m1)[:, None] + s1) > (np.arange(m2)[None, :] + s2)
    gx, gy = np.nonzero(tri)
    assert np.array_equal(d["counts"][gx, gy], pb["counts"][gx, gy]), "cell counts differ"
    assert np.array_equal(d["df1"][gx, gy], pb["df1"][gx, gy])
    assert np.array_equal(d["df2"][gx, gy], pb["df2"][gx, gy])
    d1, d2 = pb["df1"][gx, gy], pb["df2"][gx, gy]
    e = parity.f_excess(d["F"][gx, gy], pb["F"][gx, gy], d1, d2, F_TOL)
    assert e.max() <= 1.0, "F error %.3g x its bound" % e.max()
    if test == "i":
        e2 = parity.f_excess(d["F2"][gx, gy], pb["F2"][gx, gy], d1, d2, F_TOL)
        assert e2.max() <= 1.0, "F2 error %.3g x its bound" % e2.max()
    # hits: against B (FP64 decisions) and A (the reference's own kernel and order)
    excl = parity.near_threshold(pb, block, t1, t2, test, TOL_SET)
    ok, msg = parity.compare_hit_lists(got, hb, excl)
    assert ok, "vs FP64 oracle: " + msg
    if check_ref and oracles.have_ref():
        ha, ta = oracles.ref_scan_block(gp, nid, phen, block, test=test, safe=safe, chunk=chunk, t1=t1, t2=t2,
                                        nthreads=8)
        ok, msg = parity.compare_hit_lists(got, ha, excl)
        assert ok, "vs reference kernels: " + msg
        both = {k: i for i, k in enumerate(parity.pair_key(ha))}
        idx = [(i, both[k]) for i, k in enumerate(parity.pair_key(got)) if k in both]
        if idx:
            gi, ri = np.array(idx).T
            assert np.array_equal(got["df1"][gi], ha["df1"][ri])
            assert np.array_equal(got["df2"][gi], ha["df2"][ri])
    if len(got):
        assert parity.f_errors(got, pb, block, F_TOL).max() <= 1.0
    return got


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("test,safe", [("f", 0), ("i", 0), ("f", 1), ("i", 1)])
def test_single_chromosome(gpu_ctx, form, test, safe):
    codes, gp, phen = _data(500, 400, seed=21)
    t1 = synth.f_threshold(8, 491, 1e-3)
    t2 = synth.f_threshold(4, 491, 1e-3)
    got = _check_block(gpu_ctx, codes, gp, phen, (0, 400, 0, 400), test, safe, t1, t2, form)
    assert len(got) > 0


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_all_pairs_threshold_off(gpu_ctx, form):
    """Threshold -inf: every pair with a finite F is a hit, in reference order."""
    codes, gp, phen = _data(333, 250, seed=5)
    got = _check_block(gpu_ctx, codes, gp, phen, (0, 250, 0, 250), "i", 0, -1e30, -1e30, form)
    assert len(got) > 20000


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("nid", [7, 16, 31, 32, 33, 100, 129])
def test_ragged_individuals(gpu_ctx, form, nid):
    """remain-only, remain == 0 and word-boundary individual counts (readplink.c:1090-1098)."""
    codes, gp, phen = _data(nid, 90, seed=100 + nid, miss_g=0.05, miss_p=0.1)
    _check_block(gpu_ctx, codes, gp, phen, (0, 90, 0, 90), "i", 0, 1.0, 1.0, form)


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_uneven_chromosomes(gpu_ctx, form):
    """Three chromosome blocks of uneven sizes in perform_scan's (i, j <= i) order."""
    sizes = [70, 131, 45]
    nid = 260
    codes, gp, phen = _data(nid, sum(sizes), seed=9)
    starts = np.cumsum([0] + sizes[:-1])
    blocks = [(int(starts[i]), sizes[i], int(starts[j]), sizes[j]) for i in range(3) for j in range(i + 1)]
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    gpu_ctx.load_packed(gp, nid)
    gpu_ctx.set_phenotype(phen)
    opts = capi.default_opts(test="f", t1=t1, form=form, chunk=32)
    got, total, ex = gpu_ctx.scan(blocks, opts, want_blocks=True)
    off = 0
    for bi, blk in enumerate(blocks):
        mine = got[ex["block"] == bi]
        assert np.all(np.diff(np.nonzero(ex["block"] == bi)[0]) == 1), "blocks must be contiguous"
        hb, tb, pb = oracles.oracle_scan_block(codes, phen, blk, test="f", chunk=32, t1=t1, per_pair=True)
        excl = parity.near_threshold(pb, blk, t1, 0, "f", TOL_SET)
        ok, msg = parity.compare_hit_lists(mine, hb, excl)
        assert ok, "block %d: %s" % (bi, msg)
        if oracles.have_ref():
            ha, _ = oracles.ref_scan_block(gp, nid, phen, blk, test="f", chunk=32, t1=t1, nthreads=8)
            ok, msg = parity.compare_hit_lists(mine, ha, excl)
            assert ok, "block %d vs reference: %s" % (bi, msg)
        off += len(mine)
    assert off == total


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_monomorphic_and_missing_snps(gpu_ctx, form):
    """All-one-genotype SNPs (nfac small, df1 == 0 pairs) and an all-missing SNP."""
    nid, nsnp = 120, 40
    codes, gp, phen = _data(nid, nsnp, seed=77)
    codes[3, :] = 0
    codes[4, :] = 0
    codes[5, :] = 2
    codes[6, :] = 3
    codes[7, ::2] = 3
    gp = synth.pack(codes)
    got = _check_block(gpu_ctx, codes, gp, phen, (0, nsnp, 0, nsnp), "f", 0, -1e30, 0, form)
    bad = [(a, b) for a, b in parity.pair_key(got) if 6 in (a, b)]
    assert not bad, "an all-missing SNP cannot produce a finite F"


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_chunk_order(gpu_ctx, form):
    """The -i iteration size changes the output order exactly as in the reference."""
    codes, gp, phen = _data(200, 300, seed=3)
    for chunk in (16, 48, 128, 512):
        _check_block(gpu_ctx, codes, gp, phen, (0, 300, 0, 300), "f", 0, 2.0, 0, form, chunk=chunk)


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_overflow_reports_total(gpu_ctx, form):
    codes, gp, phen = _data(100, 120, seed=4)
    gpu_ctx.load_packed(gp, 100)
    gpu_ctx.set_phenotype(phen)
    opts = capi.default_opts(test="f", t1=-1e30, form=form)
    got, total, ex = gpu_ctx.scan([(0, 120, 0, 120)], opts, cap=100)
    assert ex["status"] == capi.EPI_E_OVERFLOW
    assert len(got) == 100 and total > 100
    full, total2, _ = gpu_ctx.scan([(0, 120, 0, 120)], opts, cap=1 << 20)
    assert total2 == total
    assert np.array_equal(got, full[:100])
