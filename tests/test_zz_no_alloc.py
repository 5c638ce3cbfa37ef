"""The allocation-free entry point, epi_scan_block_noalloc.

It serves callers that cannot allocate GPU memory while they run: a service that forbids
cudaMalloc once it has started (an allocation can stall or fail under memory pressure at the
worst moment), or a framework that hands out device memory only from its own pool. Such a
caller passes device buffers for every input and output; the scan's working memory is a
fixed array inside the library.

This test provides those buffers from torch, calls the entry point through the C ABI twice in
a row on the same inputs, and checks both results against the FP64 oracle and against the
ordinary entry point, epi_scan (plain popcount form), on the same data: the same hits once
sorted by pair (pairs within the parity tests' threshold neighbourhood excepted), df exact,
F and F2 within the parity tests' tolerance, and the block's largest F. The second call must
not see the first call's counts, since every call shares the fixed array. Cases: a block on
the diagonal and blocks at non-zero offsets, individual counts with and without a partial
packed word (512, 600, 4,097), phenotypes in units of 1e20 and 1e-20, and more hits than the
output holds. The file is named to run last; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu

F_TOL = 1e-5
TOL_SET = 1e-4


def _noalloc(torch, gp_dev, nid, nsnp, phen_dev, block, opts, cap, expect=capi.EPI_OK):
    lib = capi.load()
    hits = torch.zeros((max(cap, 1), 6), dtype=torch.int32, device="cuda")
    nhits = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    maxf = torch.zeros(2, dtype=torch.float32, device="cuda")
    b = capi.Block(*block)
    torch.cuda.synchronize()
    st = lib.epi_scan_block_noalloc(ctypes.c_void_p(gp_dev.data_ptr()), nid, nsnp,
                                    ctypes.c_void_p(phen_dev.data_ptr()), ctypes.byref(b), ctypes.byref(opts),
                                    ctypes.c_void_p(hits.data_ptr()), cap, ctypes.c_void_p(nhits.data_ptr()),
                                    ctypes.c_void_p(maxf.data_ptr()), None)
    assert st == expect, "epi_scan_block_noalloc returned %d, expected %d" % (st, expect)
    n = int(nhits.item())
    rows = hits[:min(n, cap)].cpu().numpy().copy().view(capi.HIT_DTYPE).reshape(-1)
    return rows, n, maxf.cpu().numpy()


def _by_pair(h):
    return h[np.lexsort((h["snp2"], h["snp1"]))]


def _check_against(got, ref, near, nsnp, test, what):
    """Hit set, df and F of `got` against `ref` (both sorted by pair)."""
    ok, msg = parity.compare_hit_lists(got, ref, near)
    assert ok, "%s: %s" % (what, msg)
    ka_key = got["snp1"].astype(np.int64) * nsnp + got["snp2"]
    kb_key = ref["snp1"].astype(np.int64) * nsnp + ref["snp2"]
    common = np.intersect1d(ka_key, kb_key)
    ka, kb = np.isin(ka_key, common), np.isin(kb_key, common)
    a, b = got[ka], ref[kb]
    assert np.array_equal(a["df1"], b["df1"]) and np.array_equal(a["df2"], b["df2"]), what
    assert parity.f_excess(a["F"], b["F"], b["df1"], b["df2"], F_TOL).max(initial=0) <= 1.0, what
    if test == "i":
        assert parity.f_excess(a["F2"], b["F2"], b["df1"], b["df2"], F_TOL).max(initial=0) <= 1.0, what


CASES = [
    # id, nid, nsnp, block (start1, size1, start2, size2), test, safe, phenotype scale
    ("offset_n600_i", 600, 320, (180, 140, 40, 120), "i", 0, 1.0),
    ("diag_n512_safe_f", 512, 200, (0, 200, 0, 200), "f", 1, 1.0),
    ("diag_offset_n4097_i", 4097, 260, (60, 150, 60, 150), "i", 0, 1.0),
    ("scale_1e20_i", 600, 160, (0, 160, 0, 160), "i", 0, 1e20),
    ("scale_1e-20_i", 600, 160, (0, 160, 0, 160), "i", 0, 1e-20),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_oracle_and_epi_scan(case):
    torch = pytest.importorskip("torch")
    _, nid, nsnp, block, test, safe, scale = case
    codes = synth.genotype_codes(nid, nsnp, seed=41 + nid)
    gp = synth.pack(codes)
    phen = synth.phenotype(nid, seed=42 + nid, miss=0.03)
    if scale != 1.0:
        keep = phen != -9.0
        phen[keep] = (phen[keep].astype(np.float64) * scale + 3.0 * scale).astype(np.float32)
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    t2 = synth.f_threshold(4, nid - 9, 1e-2)
    opts = capi.default_opts(test=test, safe=safe, t1=t1, t2=t2, form=capi.FORM_POPC)

    hb, _, pb = oracles.oracle_scan_block(codes, phen, block, test=test, safe=safe, t1=t1, t2=t2, per_pair=True)
    near = parity.near_threshold(pb, block, t1, t2, test, TOL_SET)
    s1, m1, s2, m2 = block
    tri = (np.arange(m1)[:, None] + s1) > (np.arange(m2)[None, :] + s2)
    fin = np.isfinite(pb["F"]) & tri
    oracle_max = pb["F"][fin].max()

    with capi.Context(0) as ctx:
        ctx.load_packed(gp, nid)
        ctx.set_phenotype(phen, safe=safe)
        ref, ntot, ex = ctx.scan([block], opts)
    assert ntot > 20

    gp_dev = torch.from_numpy(np.ascontiguousarray(gp)).cuda()
    phen_dev = torch.from_numpy(np.ascontiguousarray(phen)).cuda()
    for call in range(2):
        got, n, maxf = _noalloc(torch, gp_dev, nid, nsnp, phen_dev, block, opts, cap=1 << 16)
        assert n == len(got)
        got = _by_pair(got)
        _check_against(got, _by_pair(hb), near, nsnp, test, "call %d vs oracle" % (call + 1))
        _check_against(got, _by_pair(ref), near, nsnp, test, "call %d vs epi_scan" % (call + 1))
        assert abs(maxf[0] - oracle_max) <= F_TOL * max(1.0, abs(oracle_max)), (maxf[0], oracle_max)
        assert abs(maxf[0] - ex["max_f"][0]) <= F_TOL * max(1.0, abs(ex["max_f"][0]))


def test_noalloc_reports_overflow():
    """More hits than the caller's buffer: the first `cap` rows are written, the total is in
    *d_nhits and the status is EPI_E_OVERFLOW; the next call with room returns every hit."""
    torch = pytest.importorskip("torch")
    nid, nsnp = 300, 120
    codes = synth.genotype_codes(nid, nsnp, seed=71)
    gp = synth.pack(codes)
    phen = synth.phenotype(nid, seed=72, miss=0.02)
    block = (0, nsnp, 0, nsnp)
    opts = capi.default_opts(test="f", t1=0.5, form=capi.FORM_POPC)
    gp_dev = torch.from_numpy(np.ascontiguousarray(gp)).cuda()
    phen_dev = torch.from_numpy(np.ascontiguousarray(phen)).cuda()
    _, total = oracles.oracle_scan_block(codes, phen, block, test="f", t1=0.5)
    assert total > 100
    few, n, _ = _noalloc(torch, gp_dev, nid, nsnp, phen_dev, block, opts, cap=50, expect=capi.EPI_E_OVERFLOW)
    assert len(few) == 50 and abs(n - total) <= max(2, total // 1000)
    every, n2, _ = _noalloc(torch, gp_dev, nid, nsnp, phen_dev, block, opts, cap=1 << 16)
    assert n2 == n == len(every)
    keys = set(zip(every["snp1"].tolist(), every["snp2"].tolist()))
    assert set(zip(few["snp1"].tolist(), few["snp2"].tolist())) <= keys


def test_noalloc_rejects_too_many_individuals():
    lib = capi.load()
    b = capi.Block(0, 1, 0, 1)
    opts = capi.default_opts()
    dummy = ctypes.c_void_p(16)
    st = lib.epi_scan_block_noalloc(dummy, capi_max() + 1, 2, dummy, ctypes.byref(b), ctypes.byref(opts), dummy, 1,
                                    dummy, None, None)
    assert st == capi.EPI_E_UNSUPPORTED


def capi_max():
    import re
    from pathlib import Path
    text = (Path(__file__).resolve().parents[1] / "include" / "epigpu.h").read_text()
    return int(re.search(r"#define EPI_NOALLOC_MAX_NID (\d+)", text).group(1))
