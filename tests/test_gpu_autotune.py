"""Kernel variants and the autotuner.

Each form has a table of kernel variants (plain form: tile shapes -- 64 x 64 with 8 pairs per
thread, 64 x 32 with 4, 32 x 128 with 8; tensor form: operand ring depths, 8 or 12
epilogue warps, one or two producer groups, B built in shared memory or streamed from HBM).
Every variant must
give the oracle's results: counts and df exact, F within the parity bar, the same hits in the
same order (several uneven chromosome blocks, several traits with their own masks). The
autotuner times every candidate once per device, form, individual count and trait count and
keeps the fastest; epi_scan_config reports the choice and the timings."""
import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu

F_TOL = 1e-5
TOL_SET = 1e-4
N_CANDIDATES = {capi.FORM_POPC: 3, capi.FORM_TENSOR: 6}
VARIANTS = [(f, c) for f in (capi.FORM_POPC, capi.FORM_TENSOR) for c in range(1, N_CANDIDATES[f] + 1)]


@pytest.mark.parametrize("form,cand", VARIANTS,
                         ids=["%s%d" % ("popc" if f == capi.FORM_POPC else "tensor", c) for f, c in VARIANTS])
def test_every_variant_matches_oracle(gpu_ctx, form, cand):
    nid, sizes = 611, [150, 97, 201]
    codes = synth.genotype_codes(nid, sum(sizes), seed=401)
    rng = np.random.default_rng(402)
    Y = np.stack([rng.standard_normal(nid), (rng.gamma(2.0, 1.0, nid) - 2.0) / np.sqrt(2.0)], 1).astype(np.float32)
    V = np.stack([rng.random(nid) >= 0.02, rng.random(nid) >= 0.08], 1)
    gpu_ctx.load_packed(synth.pack(codes), nid)
    gpu_ctx.set_traits(Y, V)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    blocks = [(int(starts[i]), sizes[i], int(starts[j]), sizes[j]) for i in range(3) for j in range(i + 1)]
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    t2 = synth.f_threshold(4, nid - 9, 1e-2)
    opts = capi.default_opts(test="i", t1=t1, t2=t2, form=form, report_trait=-1, tile_config=cand)
    hits, total, ex = gpu_ctx.scan(blocks, opts, ntraits=2, want_blocks=True, want_traits=True)
    cfg = gpu_ctx.scan_config()
    assert "requested" in cfg and ("tensor" if form == capi.FORM_TENSOR else "plain") in cfg, cfg
    assert total == len(hits) > 100
    for t in range(2):
        phen = np.where(V[:, t], Y[:, t], np.float32(-9.0)).astype(np.float32)
        for b, blk in enumerate(blocks):
            mine = hits[(ex["trait"] == t) & (ex["block"] == b)]
            hb, _, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=t1, t2=t2, per_pair=True)
            excl = parity.near_threshold(pb, blk, t1, t2, "i", TOL_SET)
            ok, msg = parity.compare_hit_lists(mine, hb, excl)
            assert ok, "trait %d block %d: %s" % (t, b, msg)
            if len(mine):
                assert parity.f_errors(mine, pb, blk, F_TOL).max() <= 1.0
                assert parity.f_errors(mine, pb, blk, F_TOL, field="F2").max() <= 1.0
    blk = blocks[4]
    d = gpu_ctx.scan_dump(blk, capi.default_opts(test="i", t1=t1, t2=t2, form=form, tile_config=cand), trait=1)
    phen = np.where(V[:, 1], Y[:, 1], np.float32(-9.0)).astype(np.float32)
    _, _, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=t1, t2=t2, per_pair=True)
    s1, m1, s2, m2 = blk
    tri = (np.arange(m1)[:, None] + s1) > (np.arange(m2)[None, :] + s2)
    assert np.array_equal(d["counts"][tri], pb["counts"][tri])
    assert np.array_equal(d["df1"][tri], pb["df1"][tri]) and np.array_equal(d["df2"][tri], pb["df2"][tri])


@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
def test_autotuner_choice_is_reported_and_kept(gpu_ctx, form):
    nid, nsnp = 1500, 2000
    codes = synth.genotype_codes(nid, nsnp, seed=411)
    phen = synth.phenotype(nid, seed=412)
    gpu_ctx.load_packed(synth.pack(codes), nid)
    gpu_ctx.set_phenotype(phen)
    t1 = synth.f_threshold(8, nid - 9, 1e-3)
    opts = capi.default_opts(test="f", t1=t1, form=form)
    first, n1, _ = gpu_ctx.scan([(0, nsnp, 0, nsnp)], opts)
    cfg = gpu_ctx.scan_config()
    nc = N_CANDIDATES[form]
    assert "autotuned" in cfg and cfg.count(" ms") == nc, cfg
    again, n2, _ = gpu_ctx.scan([(0, nsnp, 0, nsnp)], opts)
    assert gpu_ctx.scan_config() == cfg  # kept, not tuned again
    assert n1 == n2 and np.array_equal(first, again)
    # the chosen candidate, requested by number, gives the same hits
    names = {k: None for k in range(1, nc + 1)}
    for k in names:
        gpu_ctx.scan([(0, 10, 0, 10)], capi.default_opts(test="f", t1=t1, form=form, tile_config=k))
        names[k] = gpu_ctx.scan_config().split(" (")[0]
    chosen = [k for k, v in names.items() if cfg.startswith(v)]
    assert len(chosen) == 1, (cfg, names)
    forced, n3, _ = gpu_ctx.scan([(0, nsnp, 0, nsnp)], capi.default_opts(test="f", t1=t1, form=form,
                                                                         tile_config=chosen[0]))
    assert n3 == n1 and np.array_equal(forced, first)
    with pytest.raises(capi.EpiError) as err:
        gpu_ctx.scan([(0, 10, 0, 10)], capi.default_opts(form=form, tile_config=nc + 1))
    assert err.value.status == capi.EPI_E_INVALID
