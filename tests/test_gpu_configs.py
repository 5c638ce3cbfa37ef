"""GPU parity at the shapes of the benchmark configurations, against the FP64 oracle.

  2 plain 4 df interaction scan: N = 4,000 individuals, 20,000 SNPs on 2 chromosomes
    (three chromosome blocks, one of them between the chromosomes), phenotype = N(0,1) plus
    5 planted pairs, each with a random mean-0 3x3 genotype-class effect table, 1% missing.
  4 batched permutations: N = 5,000, 50,000 SNPs, 64 phenotype columns in one scan -- column
    0 with 3 planted pairs, columns 1-63 its permutations by the reference's -p rule
    (src/main.c:336-348) -- and one shared 1% missing mask.
  5 uneven blocks, several traits: N = 8,000 over 22 chromosome blocks of 2,000 to 24,000 SNPs
    (250,000 SNPs), 8 traits (normal and standardised gamma(2,1)), each with its own 0-10%
    missingness mask, so counts are mask-weighted.

The scans run at the configurations' own sizes on the GPU (all pairs for 2 and 4; for 5 the 15
blocks between 5 of the 22 chromosomes, 1.9e9 pairs x 8 traits). The oracle cannot scan that
many pairs, so it checks what it can: sub-blocks (inside a chromosome and between two) per trait
at a threshold loose enough to give many hits -- counts and df exact, F and F2 within 1e-5,
the hit set equal away from the threshold -- every planted pair's statistics and hit decision,
and per-column maxima over a sampled block for all 64 columns.

Planted-pair power: at the configuration's effect size (0.5% of the variance per pair) and
N = 4,000, a planted pair's expected 8 df F is about 3.6 against a p = 1e-6 threshold of 5.36:
about 8% of such pairs reach it, so at that size the test asserts the oracle's decision for each
planted pair rather than recovery. Recovery itself is asserted with pairs that explain 2% of the
variance each (power above 99% per pair at p = 1e-6), in configurations 2 and 4.
"""
import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu

F_TOL = 1e-5
TOL_SET = 1e-4


def _thresholds(nid, p):
    return synth.f_threshold(8, nid - 9, p), synth.f_threshold(4, nid - 9, p)


def _chrom_blocks(sizes, chroms):
    """perform_scan's blocks (i, j <= i) over the chosen chromosomes (src/EpiOpenCL.c:1527-1540)."""
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
    return [(int(starts[i]), int(sizes[i]), int(starts[j]), int(sizes[j]))
            for a, i in enumerate(chroms) for j in chroms[:a + 1]]


def _in_block(h, blk):
    s1, m1, s2, m2 = blk
    return (h["snp1"] >= s1) & (h["snp1"] < s1 + m1) & (h["snp2"] >= s2) & (h["snp2"] < s2 + m2)


def _oracle_sub(gp, nid, phen, blk, test, t1, t2):
    """Oracle B on a sub-block of a genome held only in packed form: hits (global indices)
    and per-pair statistics."""
    s1, m1, s2, m2 = blk
    lo, hi = min(s1, s2), max(s1 + m1, s2 + m2)
    if hi - lo <= m1 + m2:  # overlapping or adjacent ranges: unpack the span
        codes = synth.unpack(gp[lo:hi], nid)
        local = (s1 - lo, m1, s2 - lo, m2)
        off1 = off2 = lo
    else:  # disjoint ranges: stack them, SNP2 range first so snp1 > snp2 still holds
        assert s1 >= s2 + m2, "disjoint sub-blocks must lie below the diagonal"
        codes = synth.unpack(np.concatenate([gp[s2:s2 + m2], gp[s1:s1 + m1]]), nid)
        local = (m2, m1, 0, m2)
        off1, off2 = s1 - m2, s2
    hb, _, pb = oracles.oracle_scan_block(codes, phen, local, test=test, t1=t1, t2=t2, per_pair=True)
    hb = hb.copy()
    hb["snp1"] += off1
    hb["snp2"] += off2
    return hb, pb


def _check_sub(got, gp, nid, phen, blk, test, t1, t2, what):
    """Hits of `got` inside `blk` against the oracle's hits of that block."""
    hb, pb = _oracle_sub(gp, nid, phen, blk, test, t1, t2)
    near = parity.near_threshold(pb, blk, t1, t2, test, TOL_SET)
    mine = got[_in_block(got, blk)]
    a = set(zip(mine["snp1"].tolist(), mine["snp2"].tolist())) - near
    b = set(zip(hb["snp1"].tolist(), hb["snp2"].tolist())) - near
    assert a == b, "%s: only GPU %s, only oracle %s" % (what, sorted(a - b)[:5], sorted(b - a)[:5])
    if len(mine):
        assert parity.f_errors(mine, pb, blk, F_TOL).max() <= 1.0, what
        if test == "i":
            assert parity.f_errors(mine, pb, blk, F_TOL, field="F2").max() <= 1.0, what
    return len(b)


def _dump_check(ctx, gp, nid, phen, blk, test, form, trait=0):
    """Counts, df and F of every pair of `blk` from the GPU dump against the oracle."""
    _, pb = _oracle_sub(gp, nid, phen, blk, test, -1e30, -1e30)
    d = ctx.scan_dump(blk, capi.default_opts(test=test, t1=-1e30, t2=-1e30, form=form), trait=trait)
    s1, m1, s2, m2 = blk
    tri = (np.arange(m1)[:, None] + s1) > (np.arange(m2)[None, :] + s2)
    assert np.array_equal(d["counts"][tri], pb["counts"][tri]), "cell counts"
    assert np.array_equal(d["df1"][tri], pb["df1"][tri]) and np.array_equal(d["df2"][tri], pb["df2"][tri])
    for f in ("F", "F2") if test == "i" else ("F",):
        e = parity.f_excess(d[f][tri], pb[f][tri], pb["df1"][tri], pb["df2"][tri], F_TOL)
        assert e.max() <= 1.0, "%s error %.3g x its bound" % (f, e.max())
    return pb


def _pair_stats(gp, nid, phen, a, b, test="i"):
    codes = synth.unpack(gp[[b, a]], nid)
    _, _, pb = oracles.oracle_scan_block(codes, phen, (1, 1, 0, 1), test=test, t1=-1e30, t2=-1e30, per_pair=True)
    return pb["F"][0, 0], pb["F2"][0, 0], pb["df1"][0, 0], pb["df2"][0, 0]


# ---------------------------------------------------------------------------------------
# configuration 2: N = 4,000, 2 x 10,000 SNPs, 8 df + 4 df, 5 planted pairs
# ---------------------------------------------------------------------------------------
NID2, SIZES2 = 4000, [10000, 10000]
PLANTED2 = [(1500, 300), (12000, 4000), (18500, 11000), (10005, 9995), (9000, 8990)]


@pytest.fixture(scope="module")
def cfg2():
    codes = synth.genotype_codes(NID2, sum(SIZES2), seed=201)
    gp = synth.pack(codes)
    spec = synth.planted_phenotype(codes, PLANTED2, seed=202, var_frac=0.005, miss=0.01)
    strong = synth.planted_phenotype(codes, PLANTED2, seed=203, var_frac=0.02, miss=0.01)
    return gp, spec, strong


@pytest.mark.parametrize("form", [capi.FORM_TENSOR, capi.FORM_POPC], ids=["tensor", "popc"])
def test_cfg2_shape(gpu_ctx, cfg2, form):
    gp, spec, strong = cfg2
    blocks = _chrom_blocks(SIZES2, [0, 1])
    t1, t2 = _thresholds(NID2, 1e-6)
    gpu_ctx.load_packed(gp, NID2)
    opts = capi.default_opts(test="i", t1=t1, t2=t2, form=form)

    # the configuration's effect size: every planted pair decided as the oracle decides it
    gpu_ctx.set_phenotype(spec)
    hits, total, ex = gpu_ctx.scan(blocks, opts, want_blocks=True)
    assert total == len(hits) and np.all(np.diff(ex["block"]) >= 0)
    got = set(zip(hits["snp1"].tolist(), hits["snp2"].tolist()))
    for a, b in PLANTED2:
        F, F2, d1, d2 = _pair_stats(gp, NID2, spec, a, b)
        is_hit = (F > t1 or F2 > t2) and d1 + 1 > 6
        near = min(abs(F - t1) / t1, abs(F2 - t2) / t2) <= TOL_SET
        assert near or ((a, b) in got) == is_hit, (a, b, F, F2)
    # one sub-block inside a chromosome and one between the chromosomes, each around a
    # planted pair, at this threshold
    for blk in [(8850, 300, 8850, 300), (11850, 300, 3850, 300)]:
        _check_sub(hits, gp, NID2, spec, blk, "i", t1, t2, "cfg2 sub-block %s" % (blk,))

    # parity at a loose threshold (many hits) on the same sub-blocks, in one launch
    l1, l2 = _thresholds(NID2, 1e-2)
    subs = [(8850, 300, 8850, 300), (11850, 300, 3850, 300)]
    loose, _, _ = gpu_ctx.scan(subs, capi.default_opts(test="i", t1=l1, t2=l2, form=form))
    n = sum(_check_sub(loose, gp, NID2, spec, blk, "i", l1, l2, "cfg2 loose %s" % (blk,)) for blk in subs)
    assert n > 500
    _dump_check(gpu_ctx, gp, NID2, spec, (11900, 120, 3900, 120), "i", form)

    # recovery: pairs explaining 2% of the variance each are all found
    gpu_ctx.set_phenotype(strong)
    hits, total, _ = gpu_ctx.scan(blocks, opts)
    got = set(zip(hits["snp1"].tolist(), hits["snp2"].tolist()))
    missing = [p for p in PLANTED2 if p not in got]
    assert not missing, missing


# ---------------------------------------------------------------------------------------
# configuration 4: N = 5,000, 50,000 SNPs, 64 columns (column 0 + 63 permutations)
# ---------------------------------------------------------------------------------------
NID4, NSNP4, T4 = 5000, 50000, 64
PLANTED4 = [(31000, 2000), (45000, 44000), (20000, 19000)]


@pytest.fixture(scope="module")
def cfg4():
    codes = synth.genotype_codes(NID4, NSNP4, seed=401)
    gp = synth.pack(codes)
    rows = {s: codes[s].copy() for p in PLANTED4 for s in p}
    del codes
    y0 = synth.planted_phenotype(rows, PLANTED4, seed=402, var_frac=0.02, miss=0.0)
    Y = np.stack([y0] + [capi.permute_phenotype(y0, p) for p in range(1, T4)], 1)
    valid = np.repeat((np.random.default_rng(403).random(NID4) >= 0.01)[:, None], T4, 1)
    return gp, Y, valid


def _masked(Y, V, t):
    return np.where(V[:, t], Y[:, t], np.float32(-9.0)).astype(np.float32)


def test_cfg4_shape(gpu_ctx, cfg4):
    gp, Y, V = cfg4
    t1, t2 = _thresholds(NID4, 1e-6)
    gpu_ctx.load_packed(gp, NID4)
    gpu_ctx.set_traits(Y, V)
    full = [(0, NSNP4, 0, NSNP4)]
    hits, total, ex = gpu_ctx.scan(full, capi.default_opts(test="f", t1=t1, form=capi.FORM_TENSOR, report_trait=0),
                                   ntraits=T4)
    assert total == len(hits)
    phen0 = _masked(Y, V, 0)
    got = set(zip(hits["snp1"].tolist(), hits["snp2"].tolist()))
    missing = [p for p in PLANTED4 if p not in got]
    assert not missing, missing
    # column-0 hits around a planted pair against the oracle
    _check_sub(hits, gp, NID4, phen0, (30900, 200, 1900, 200), "f", t1, t2, "cfg4 column 0")
    # maxima: column 0's is at least the planted pairs' F (oracle)
    top = max(_pair_stats(gp, NID4, phen0, a, b, test="f")[0] for a, b in PLANTED4)
    assert ex["max_f"][0] >= top * (1 - F_TOL)

    # per-column maxima of every column over a sampled block, against the oracle
    samp = (40000, 150, 10000, 150)
    _, _, sx = gpu_ctx.scan([samp], capi.default_opts(test="i", t1=t1, t2=t2, form=capi.FORM_TENSOR,
                                                      report_trait=-1), ntraits=T4)
    codes = synth.unpack(np.concatenate([gp[10000:10150], gp[40000:40150]]), NID4)
    for t in range(T4):
        _, _, pb = oracles.oracle_scan_block(codes, _masked(Y, V, t), (150, 150, 0, 150), test="i", t1=-1e30,
                                             t2=-1e30, per_pair=True)
        for key, name in (("F", "max_f"), ("F2", "max_f2")):
            v = pb[key][np.isfinite(pb[key])]
            assert abs(sx[name][t] - v.max()) <= F_TOL * max(1.0, v.max()), (t, key, sx[name][t], v.max())
        assert ex["max_f"][t] >= sx["max_f"][t] * (1 - F_TOL)  # full scan covers the sample
    # counts and F of a permuted column, every pair of a small block
    _dump_check(gpu_ctx, gp, NID4, _masked(Y, V, 37), (40000, 100, 10000, 100), "f", capi.FORM_TENSOR, trait=37)


# ---------------------------------------------------------------------------------------
# configuration 5: N = 8,000, 22 uneven chromosome blocks, 8 traits with their own masks
# ---------------------------------------------------------------------------------------
NID5, T5 = 8000, 8
CHROMS5 = [0, 5, 10, 15, 21]


@pytest.fixture(scope="module")
def cfg5():
    sizes = synth.uneven_block_sizes()
    gp = synth.packed_on_gpu(NID5, sum(sizes), seed=501)
    rng = np.random.default_rng(502)
    cols, vcols = [], []
    for t in range(T5):
        v = rng.standard_normal(NID5) if t % 2 == 0 else (rng.gamma(2.0, 1.0, NID5) - 2.0) / np.sqrt(2.0)
        cols.append(v.astype(np.float32))
        vcols.append(rng.random(NID5) >= 0.10 * t / (T5 - 1))  # 0% .. 10% missing
    return sizes, gp, np.stack(cols, 1), np.stack(vcols, 1)


def test_cfg5_shape(gpu_ctx, cfg5):
    sizes, gp, Y, V = cfg5
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int)
    blocks = _chrom_blocks(sizes, CHROMS5)
    assert len(blocks) == 15 and len({b[1] for b in blocks}) == 5
    t1, t2 = _thresholds(NID5, 1e-6)
    gpu_ctx.load_packed(gp, NID5)
    gpu_ctx.set_traits(Y, V)
    hits, total, ex = gpu_ctx.scan(blocks, capi.default_opts(test="f", t1=t1, form=capi.FORM_TENSOR,
                                                             report_trait=-1),
                                   ntraits=T5, want_traits=True, want_blocks=True)
    assert total == len(hits) and total > 1000
    assert np.all(np.diff(ex["trait"]) >= 0)
    for t in range(T5):
        mine = hits[ex["trait"] == t]
        assert len(mine) and ex["max_f"][t] >= mine["F"].max() * (1 - F_TOL)
        for b in np.unique(ex["block"][ex["trait"] == t]):
            assert np.all(_in_block(mine[ex["block"][ex["trait"] == t] == b], blocks[b]))

    # per trait, a sub-block inside a chromosome and one between two chromosomes, in one launch
    # at a loose threshold, against the oracle with that trait's own mask
    intra = (int(starts[10]) + 100, 250, int(starts[10]) + 100, 250)
    inter = (int(starts[21]) + 500, 250, int(starts[0]) + 7000, 250)
    l1, l2 = _thresholds(NID5, 1e-2)
    loose, _, lx = gpu_ctx.scan([intra, inter], capi.default_opts(test="i", t1=l1, t2=l2, form=capi.FORM_TENSOR,
                                                                  report_trait=-1),
                                ntraits=T5, want_traits=True)
    for t in range(T5):
        phen = _masked(Y, V, t)
        mine = loose[lx["trait"] == t]
        n = sum(_check_sub(mine, gp, NID5, phen, blk, "i", l1, l2, "cfg5 trait %d %s" % (t, blk))
                for blk in (intra, inter))
        assert n > 100
    _dump_check(gpu_ctx, gp, NID5, _masked(Y, V, 7), (int(starts[15]) + 10, 90, int(starts[5]) + 20, 90), "i",
                capi.FORM_TENSOR, trait=7)
