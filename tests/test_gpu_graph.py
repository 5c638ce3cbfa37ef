"""The scan's device part under captured CUDA graphs.

epi_scan captures its device work -- scan-state reset, schedule upload, the persistent pair
kernel between the timing events, counter and maxima readback -- as a CUDA graph, and a repeat
of the same scan shape replays it with one launch (the reference instead blocks on every
chunk launch, src/EpiOpenCL.c:1576-1607). Replayed scans must give exactly what an uncaptured
launch gives (no_graph = 1): hits in order, F values, maxima; a new shape is captured anew; the
rescan after the device hit buffer grows is launched directly. Both forms, several uneven
chromosome blocks in one launch."""
import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu


def _same(a, b):
    (h1, n1, e1), (h2, n2, e2) = a, b
    assert n1 == n2 and np.array_equal(h1, h2)
    assert np.array_equal(e1["max_f"], e2["max_f"]) and np.array_equal(e1["max_f2"], e2["max_f2"])
    assert np.array_equal(e1["block"], e2["block"])


@pytest.mark.parametrize("form", [capi.FORM_TENSOR, capi.FORM_POPC], ids=["tensor", "popc"])
def test_replayed_graph_equals_direct_launch(gpu_ctx, form):
    nid, sizes = 900, [300, 170, 230]
    codes = synth.genotype_codes(nid, sum(sizes), seed=301)
    phen = synth.phenotype(nid, seed=302)
    gpu_ctx.load_packed(synth.pack(codes), nid)
    gpu_ctx.set_phenotype(phen)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    blocks = [(int(starts[i]), sizes[i], int(starts[j]), sizes[j]) for i in range(3) for j in range(i + 1)]
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    t2 = synth.f_threshold(4, nid - 9, 1e-2)
    direct = gpu_ctx.scan(blocks, capi.default_opts(test="i", t1=t1, t2=t2, form=form, no_graph=1),
                          want_blocks=True)
    opts = capi.default_opts(test="i", t1=t1, t2=t2, form=form)
    runs = [gpu_ctx.scan(blocks, opts, want_blocks=True) for _ in range(3)]  # capture, then replays
    for r in runs:
        _same(r, direct)
        ms, pairs, launches, used = gpu_ctx.last_timing()
        assert ms > 0 and used == form and launches == 2
    assert direct[1] > 50
    # the hits of one block against the oracle
    hits, _, ex = runs[-1]
    blk = blocks[3]
    hb, _, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=t1, t2=t2, per_pair=True)
    near = parity.near_threshold(pb, blk, t1, t2, "i", 1e-4)
    ok, msg = parity.compare_hit_lists(hits[ex["block"] == 3], hb, near)
    assert ok, msg

    # a different shape (fewer blocks) is captured anew; then the first shape again
    sub = gpu_ctx.scan(blocks[:2], opts, want_blocks=True)
    _same(sub, gpu_ctx.scan(blocks[:2], capi.default_opts(test="i", t1=t1, t2=t2, form=form, no_graph=1),
                            want_blocks=True))
    _same(gpu_ctx.scan(blocks, opts, want_blocks=True), direct)


def test_hit_buffer_regrow_falls_back_to_direct_launch():
    """More hits than a new context's device hit buffer holds (2^20): the buffer grows and the
    scan runs again directly; later scans of that shape are captured with the new buffer.
    Every pair is a hit here (threshold below any F)."""
    nid, nsnp = 300, 1600
    codes = synth.genotype_codes(nid, nsnp, seed=311)
    blk = [(0, nsnp, 0, nsnp)]
    opts = capi.default_opts(test="f", t1=-1.0, form=capi.FORM_TENSOR)
    with capi.Context(0) as ctx:
        ctx.load_packed(synth.pack(codes), nid)
        ctx.set_phenotype(synth.phenotype(nid, seed=312))
        first = ctx.scan(blk, opts, cap=1 << 21, want_blocks=True)
        assert (1 << 20) < first[1] <= nsnp * (nsnp - 1) // 2
        again = ctx.scan(blk, opts, cap=1 << 21, want_blocks=True)
        _same(first, again)
        direct = ctx.scan(blk, capi.default_opts(test="f", t1=-1.0, form=capi.FORM_TENSOR, no_graph=1),
                          cap=1 << 21, want_blocks=True)
        _same(first, direct)
