"""Edge inputs: empty scans (no blocks, zero-size blocks, blocks without a pair), a single
individual, and more individuals than the plain form's 16-bit counters allow (the tensor
form's exact int32 counts against the FP64 oracle; the plain form refuses)."""
import numpy as np
import pytest

from epigpu_b200 import capi, synth
from test_gpu_parity import FORMS, FORM_IDS, _check_block, _data

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_empty_scans(gpu_ctx, form):
    codes, gp, phen = _data(50, 20, seed=91)
    gpu_ctx.load_packed(gp, 50)
    gpu_ctx.set_phenotype(phen)
    opts = capi.default_opts(test="i", t1=1.0, t2=1.0, form=form)
    hits, total, _ = gpu_ctx.scan([], opts)
    assert total == 0 and len(hits) == 0
    for blk in [(0, 0, 0, 10), (5, 10, 5, 0), (3, 1, 3, 1), (3, 1, 4, 1)]:
        hits, total, _ = gpu_ctx.scan([blk], opts)
        assert total == 0, blk
    # empty blocks around a real one change nothing
    ref, rtotal, _ = gpu_ctx.scan([(0, 20, 0, 20)], opts)
    got, total, ex = gpu_ctx.scan([(0, 0, 0, 10), (0, 20, 0, 20), (3, 1, 3, 1)], opts, want_blocks=True)
    assert rtotal > 0 and total == rtotal
    assert np.array_equal(got[["snp1", "snp2", "df1", "df2"]], ref[["snp1", "snp2", "df1", "df2"]])
    assert np.all(ex["block"] == 1)


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
def test_single_individual(gpu_ctx, form):
    """Every pair holds at most one individual: counts exact, df1 = 0, F undefined, no hit."""
    codes, gp, phen = _data(1, 12, seed=92, miss_g=0.0, miss_p=0.0)
    gpu_ctx.load_packed(gp, 1)
    gpu_ctx.set_phenotype(phen)
    opts = capi.default_opts(test="f", t1=1.0, form=form)
    hits, total, _ = gpu_ctx.scan([(0, 12, 0, 12)], opts)
    assert total == 0
    d = gpu_ctx.scan_dump((0, 12, 0, 12), opts)
    tri = np.tril(np.ones((12, 12), bool), -1)
    assert np.all(d["counts"][tri].sum(-1) == 1)
    assert np.all(d["df1"][tri] == 0)


def test_more_individuals_than_16_bit_counts(gpu_ctx):
    nid = 70001
    codes, gp, phen = _data(nid, 20, seed=93)
    # the reference's own kernel counts in unsigned short and overflows here: FP64 oracle only
    _check_block(gpu_ctx, codes, gp, phen, (0, 20, 0, 20), "i", 0, 3.0, 3.0, capi.FORM_TENSOR, check_ref=False)
    opts = capi.default_opts(test="i", form=capi.FORM_POPC)
    with pytest.raises(capi.EpiError) as e:
        gpu_ctx.scan([(0, 20, 0, 20)], opts)
    assert e.value.status == capi.EPI_E_UNSUPPORTED
