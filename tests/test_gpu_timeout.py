"""Failure detection of the tensor form's device-side waits, without a GPU fault.

Every wait of the tensor kernel's pipeline (TMA arrivals, MMA completions, the CTA pair's
handshakes) gives up after a limit and the scan returns EPI_E_TIMEOUT instead of hanging;
the reference reports its own device errors through ereport (src/EpiOpenCL.c:1159-1177).
Here the limit is set short (20 ms) and the test hook EPI_DEBUG_STALL makes the first CTA
pair's MMA issuer wait on a barrier that nothing arrives at, so that wait runs out. The
scan must return the timeout status within a bounded time, and the same context must then
scan correctly (hits against the FP64 oracle)."""
import time

import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu


def test_stalled_wait_times_out_and_context_recovers(gpu_ctx):
    nid, nsnp = 1000, 240
    codes = synth.genotype_codes(nid, nsnp, seed=91)
    gp = synth.pack(codes)
    phen = synth.phenotype(nid, seed=92, miss=0.02)
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    t2 = synth.f_threshold(4, nid - 9, 1e-2)
    blk = (0, nsnp, 0, nsnp)
    gpu_ctx.load_packed(gp, nid)
    gpu_ctx.set_phenotype(phen)

    stalled = capi.default_opts(test="i", t1=t1, t2=t2, form=capi.FORM_TENSOR, wait_limit_ms=20,
                                debug=capi.DEBUG_STALL)
    t = time.perf_counter()
    with pytest.raises(capi.EpiError) as err:
        gpu_ctx.scan([blk], stalled)
    elapsed = time.perf_counter() - t
    assert err.value.status == capi.EPI_E_TIMEOUT, str(err.value)
    assert elapsed < 10.0, elapsed

    # the context is still usable: a normal scan gives the oracle's hits
    hb, _, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=t1, t2=t2, per_pair=True)
    near = parity.near_threshold(pb, blk, t1, t2, "i", 1e-4)
    for limit in (0, 20):  # default limit, and the short limit without the stall
        opts = capi.default_opts(test="i", t1=t1, t2=t2, form=capi.FORM_TENSOR, wait_limit_ms=limit)
        got, total, _ = gpu_ctx.scan([blk], opts)
        assert total == len(got) > 10
        ok, msg = parity.compare_hit_lists(got, hb, near)
        assert ok, msg
        assert parity.f_errors(got, pb, blk, 1e-5).max() <= 1.0


def test_wait_limit_is_validated(gpu_ctx):
    nid, nsnp = 300, 40
    codes = synth.genotype_codes(nid, nsnp, seed=93)
    gpu_ctx.load_packed(synth.pack(codes), nid)
    gpu_ctx.set_phenotype(synth.phenotype(nid, seed=94))
    for bad in (dict(wait_limit_ms=-1), dict(debug=7)):
        with pytest.raises(capi.EpiError) as err:
            gpu_ctx.scan([(0, nsnp, 0, nsnp)], capi.default_opts(form=capi.FORM_TENSOR, **bad))
        assert err.value.status == capi.EPI_E_INVALID
    got, total, _ = gpu_ctx.scan([(0, nsnp, 0, nsnp)], capi.default_opts(form=capi.FORM_TENSOR, t1=1.0))
    assert total == len(got)
    assert np.all(got["snp1"] > got["snp2"])
