"""F accuracy at the headline's individual count (N = 10,000): both GPU forms against
the FP64 oracle on every pair of a seeded 600-SNP block (179,700 pairs), 8 df and 4 df.
Reports max and median relative error over the pairs with F >= 1 and the max absolute
error below; the bar is 1e-5 relative (absolute under F = 1; times kappa = SSY/SSW, ~1 at
this N). Cell counts must match exactly on every pair."""
import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu

NID, NSNP = 10000, 600


@pytest.fixture(scope="module")
def data():
    codes = synth.genotype_codes(NID, NSNP, seed=31)
    phen = synth.phenotype(NID, seed=32, miss=0.01)
    hb, tb, pb = oracles.oracle_scan_block(codes, phen, (0, NSNP, 0, NSNP), test="i", t1=-1e30, t2=-1e30,
                                           per_pair=True)
    return codes, synth.pack(codes), phen, pb


@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
def test_f_error_at_n10000(gpu_ctx, data, form):
    codes, gp, phen, pb = data
    gpu_ctx.load_packed(gp, NID)
    gpu_ctx.set_phenotype(phen)
    opts = capi.default_opts(test="i", t1=-1e30, t2=-1e30, form=form)
    d = gpu_ctx.scan_dump((0, NSNP, 0, NSNP), opts)
    tri = np.tril(np.ones((NSNP, NSNP), bool), -1)
    assert np.array_equal(d["counts"][tri], pb["counts"][tri])
    assert np.array_equal(d["df1"][tri], pb["df1"][tri]) and np.array_equal(d["df2"][tri], pb["df2"][tri])
    out = {}
    for field in ("F", "F2"):
        ref = pb[field][tri]
        got = d[field][tri].astype(np.float64)
        big = np.abs(ref) >= 1.0
        rel = oracles.rel_err(got[big], ref[big])
        absl = np.abs(got[~big] - ref[~big])
        out[field] = (float(rel.max()), float(np.median(rel)), int(big.sum()), float(absl.max()))
        assert parity.f_excess(got, ref, pb["df1"][tri], pb["df2"][tri], 1e-5).max() <= 1.0
        assert rel.max() <= 1e-5 and absl.max() <= 1e-5
    print("\nF error vs FP64, form %d, N=%d, %d pairs: 8df rel max %.3g median %.3g (%d pairs F>=1), abs max "
          "%.3g below; 4df rel max %.3g median %.3g (%d pairs), abs max %.3g below"
          % (form, NID, tri.sum(), *out["F"], *out["F2"]))


@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
def test_f_error_low_call_rate_individuals(gpu_ctx, form):
    """Missingness concentrated in a few individuals (48 of 2,000 miss half of all SNPs, the
    rest 0.5%), so most pairs share individuals missing at both SNPs, with a skewed trait
    and one far outlier (a large y^2 range). Every pair within the 1e-5 bar, counts exact."""
    nid, nsnp = 2000, 300
    rng = np.random.default_rng(61)
    codes = synth.genotype_codes(nid, nsnp, seed=62, miss=0.005)
    low = rng.choice(nid, 48, replace=False)
    codes[:, low] = np.where(rng.random((nsnp, low.size)) < 0.5, 3, codes[:, low])
    y = ((rng.gamma(1.5, 1.0, nid) - 1.5)).astype(np.float32)
    y[low[0]] = 25.0
    phen = np.where(rng.random(nid) < 0.02, np.float32(-9.0), y).astype(np.float32)
    blk = (0, nsnp, 0, nsnp)
    hb, tb, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=-1e30, t2=-1e30, per_pair=True)
    gpu_ctx.load_packed(synth.pack(codes), nid)
    gpu_ctx.set_phenotype(phen)
    d = gpu_ctx.scan_dump(blk, capi.default_opts(test="i", t1=-1e30, t2=-1e30, form=form))
    tri = np.tril(np.ones((nsnp, nsnp), bool), -1)
    assert np.array_equal(d["counts"][tri], pb["counts"][tri])
    for field in ("F", "F2"):
        ref, got = pb[field][tri], d[field][tri].astype(np.float64)
        assert parity.f_excess(got, ref, pb["df1"][tri], pb["df2"][tri], 1e-5).max() <= 1.0, field


@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
def test_hits_low_call_rate_individuals(gpu_ctx, form):
    """The same missingness pattern through the screened scan path (no dump): thresholds at
    the oracle's 99th and 99.5th percentiles put thousands of pairs near them, and the pairs
    sharing several individuals missing at both SNPs (one an outlier) must still give the
    oracle's hit list. The tensor form screens with a lower bound of the pair's sum of
    squares and takes the exact one only for candidates."""
    nid, nsnp = 2000, 300
    rng = np.random.default_rng(61)
    codes = synth.genotype_codes(nid, nsnp, seed=62, miss=0.005)
    low = rng.choice(nid, 48, replace=False)
    codes[:, low] = np.where(rng.random((nsnp, low.size)) < 0.5, 3, codes[:, low])
    y = ((rng.gamma(1.5, 1.0, nid) - 1.5)).astype(np.float32)
    y[low[0]] = 25.0
    phen = np.where(rng.random(nid) < 0.02, np.float32(-9.0), y).astype(np.float32)
    blk = (0, nsnp, 0, nsnp)
    _, _, pb0 = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=-1e30, t2=-1e30, per_pair=True)
    tri = np.tril(np.ones((nsnp, nsnp), bool), -1)
    t1 = float(np.quantile(pb0["F"][tri], 0.99))
    t2 = float(np.quantile(pb0["F2"][tri], 0.995))
    hb, _, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=t1, t2=t2, per_pair=True)
    near = parity.near_threshold(pb, blk, t1, t2, "i", 1e-4)
    gpu_ctx.load_packed(synth.pack(codes), nid)
    gpu_ctx.set_phenotype(phen)
    got, total, _ = gpu_ctx.scan([blk], capi.default_opts(test="i", t1=t1, t2=t2, form=form))
    assert total > 400
    ok, msg = parity.compare_hit_lists(got, hb, near)
    assert ok, msg


@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
@pytest.mark.parametrize("test", ["f", "i"])
def test_near_perfect_fit_is_a_hit(gpu_ctx, form, test):
    """A phenotype almost fully determined by one SNP pair's 3x3 genotype cells (noise 1e-6
    of the cell effects): its F is ~1e12, SSW is a 1e-12 fraction of SSY, and a single-precision
    screen of that pair would see only rounding noise in SSW. The pair must be a hit in both
    forms, as in the FP64 oracle, and the hit lists must agree."""
    nid, nsnp, pi, pj = 500, 24, 17, 5
    codes = synth.genotype_codes(nid, nsnp, seed=71, miss=0.0)
    rng = np.random.default_rng(72)
    effect = rng.standard_normal((3, 3))
    y = (effect[codes[pi], codes[pj]] + 1e-6 * rng.standard_normal(nid)).astype(np.float32)
    t1 = synth.f_threshold(8, nid - 9, 1e-6)
    t2 = synth.f_threshold(4, nid - 9, 1e-6)
    blk = (0, nsnp, 0, nsnp)
    gpu_ctx.load_packed(synth.pack(codes), nid)
    gpu_ctx.set_phenotype(y)
    hits, total, ex = gpu_ctx.scan([blk], capi.default_opts(test=test, t1=t1, t2=t2, form=form))
    hb, tb, pb = oracles.oracle_scan_block(codes, y, blk, test=test, t1=t1, t2=t2, per_pair=True)
    assert pb["F"][pi, pj] > 1e9
    assert any(int(h["snp1"]) == pi and int(h["snp2"]) == pj for h in hits), "the fitted pair is missing"
    excl = parity.near_threshold(pb, blk, t1, t2, test, 1e-4)
    ok, msg = parity.compare_hit_lists(hits, hb, excl)
    assert ok, msg


@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
@pytest.mark.parametrize("scale", [1e20, 1e-20], ids=["1e20", "1e-20"])
def test_phenotype_scale(gpu_ctx, form, scale):
    """F does not depend on the trait's units: a trait in units of 1e20 (squares beyond the
    single-precision range) or 1e-20 (squares below it) gives the same hits and F as the FP64
    oracle. The reference's float32 kernel overflows or underflows here, so only the FP64
    oracle is compared."""
    from test_gpu_parity import _check_block, _data
    codes, gp, phen = _data(800, 60, seed=95)
    scaled = np.where(phen == -9.0, np.float32(-9.0), phen * np.float32(scale)).astype(np.float32)
    t1 = synth.f_threshold(8, 800 - 9, 1e-2)
    t2 = synth.f_threshold(4, 800 - 9, 1e-2)
    got = _check_block(gpu_ctx, codes, gp, scaled, (0, 60, 0, 60), "i", 0, t1, t2, form, check_ref=False)
    assert len(got) > 0
