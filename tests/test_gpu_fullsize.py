"""The tensor form at the headline's full size (N = 10,000 individuals, M = 100,000 SNPs,
8 df + 4 df, thresholds at p = 1e-6: 4,999,950,000 pairs), checked through properties that do
not need the oracle to scan every pair:
- every sampled hit is a hit of the FP64 oracle, with F and F2 within the parity bar;
- no pair that the oracle finds in two 300 x 300 sub-blocks (one on the diagonal) is missing;
- the reported maxima are at least the largest hit's F and F2, whose F matches the oracle;
- a second scan returns the identical hit list."""
import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu

NID, NSNP = 10000, 100000
F_TOL = 1e-5
TOL_SET = 1e-4


# planted additive x additive interactions (no marginal effect): one in each checked
# sub-block and one at the far corner of the triangle
PLANTED = [(70100, 20150), (50200, 50050), (99999, 1)]


@pytest.fixture(scope="module")
def full():
    codes = synth.genotype_codes(NID, NSNP, seed=81)
    phen = synth.phenotype(NID, seed=82, miss=0.01)
    ok = phen != -9.0
    for a, b in PLANTED:
        u = [np.where(codes[s] < 3, codes[s].astype(np.float64), np.nan) for s in (a, b)]
        u = [x - np.nanmean(x) for x in u]
        w = np.nan_to_num(u[0] * u[1])
        phen[ok] += (0.15 * w / w[ok].std())[ok].astype(np.float32)
    t1 = synth.f_threshold(8, NID - 9, 1e-6)
    t2 = synth.f_threshold(4, NID - 9, 1e-6)
    return codes, synth.pack(codes), phen, t1, t2


def _pair_oracle(codes, phen, s1, s2):
    _, _, pb = oracles.oracle_scan_block(codes, phen, (int(s1), 1, int(s2), 1), test="i", t1=-1e30, t2=-1e30,
                                         per_pair=True)
    return pb["F"][0, 0], pb["F2"][0, 0], pb["df1"][0, 0], pb["df2"][0, 0]


def test_full_size_scan_properties(gpu_ctx, full):
    codes, gp, phen, t1, t2 = full
    gpu_ctx.load_packed(gp, NID)
    gpu_ctx.set_phenotype(phen)
    opts = capi.default_opts(test="i", t1=t1, t2=t2, form=capi.FORM_TENSOR)
    blocks = [(0, NSNP, 0, NSNP)]
    hits, total, ex = gpu_ctx.scan(blocks, opts)
    assert total == len(hits) and 1000 < total < 100000, total
    assert np.all(hits["snp1"] > hits["snp2"])

    # sampled hits against the FP64 oracle
    rng = np.random.default_rng(83)
    for h in hits[rng.choice(len(hits), 200, replace=False)]:
        F, F2, d1, d2 = _pair_oracle(codes, phen, h["snp1"], h["snp2"])
        assert (int(h["df1"]), int(h["df2"])) == (d1, d2)
        kap = parity.kappa(F, d1, d2)
        assert abs(h["F"] - F) <= F_TOL * kap * max(1.0, abs(F)), (h, F)
        assert abs(h["F2"] - F2) <= F_TOL * kap * max(1.0, abs(F2)), (h, F2)
        near = min(abs(F - t1) / t1, abs(F2 - t2) / t2) <= TOL_SET
        assert near or ((F > t1 or F2 > t2) and d1 + 1 > 6), (h, F, F2, d1)

    got = set(zip(hits["snp1"].tolist(), hits["snp2"].tolist()))
    for pair in PLANTED:
        assert pair in got, pair

    # no oracle hit missing in two sub-blocks (each holds a planted pair)
    for blk in [(70000, 300, 20000, 300), (50000, 300, 50000, 300)]:
        hb, _, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=t1, t2=t2, per_pair=True)
        excl = parity.near_threshold(pb, blk, t1, t2, "i", TOL_SET)
        s1, m1, s2, m2 = blk
        mine = {k for k in got if s1 <= k[0] < s1 + m1 and s2 <= k[1] < s2 + m2} - excl
        ref = set(zip(hb["snp1"].tolist(), hb["snp2"].tolist())) - excl
        assert mine == ref, (sorted(mine - ref)[:5], sorted(ref - mine)[:5])

    # maxima (over every valid pair, hits or not): at least the largest hit's F and F2, and
    # the largest hit's F is the oracle's
    top = hits[np.argmax(hits["F"])]
    F, F2, d1, d2 = _pair_oracle(codes, phen, top["snp1"], top["snp2"])
    assert abs(top["F"] - F) <= F_TOL * parity.kappa(F, d1, d2) * max(1.0, F)
    assert ex["max_f"][0] >= top["F"] * (1 - F_TOL)
    assert ex["max_f2"][0] >= hits["F2"].max() * (1 - F_TOL)

    # deterministic
    again, total2, _ = gpu_ctx.scan(blocks, opts)
    assert total2 == total and np.array_equal(again, hits)
