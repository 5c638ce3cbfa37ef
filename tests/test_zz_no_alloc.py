"""The allocation-free entry point, epi_scan_block_noalloc, against the ordinary one.

It serves callers that cannot allocate GPU memory while they run (a service that forbids
cudaMalloc after start-up, a framework that hands out device memory from its own pool):
they pass device buffers for every input and output, and the scan's working memory is a
fixed array inside the library. This test provides those buffers from torch, calls the
entry point through the C ABI twice in a row on the same inputs, and checks both results
against epi_scan (plain popcount form) on the same data: the same hits once sorted by pair
(pairs within the parity tests' threshold neighbourhood excepted), df exact, F and the
block's largest F within the parity tests' tolerance. The second call must not see the
first call's counts, since every call shares the fixed array. The file is named to run
last; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import parity
from epigpu_b200 import capi, synth

pytestmark = pytest.mark.gpu

F_TOL = 1e-5
TOL_SET = 1e-4


def _noalloc(torch, gp_dev, nid, nsnp, phen_dev, block, opts, cap):
    lib = capi.load()
    hits = torch.zeros((cap, 6), dtype=torch.int32, device="cuda")
    nhits = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    maxf = torch.zeros(2, dtype=torch.float32, device="cuda")
    b = capi.Block(*block)
    torch.cuda.synchronize()
    st = lib.epi_scan_block_noalloc(ctypes.c_void_p(gp_dev.data_ptr()), nid, nsnp,
                                    ctypes.c_void_p(phen_dev.data_ptr()), ctypes.byref(b), ctypes.byref(opts),
                                    ctypes.c_void_p(hits.data_ptr()), cap, ctypes.c_void_p(nhits.data_ptr()),
                                    ctypes.c_void_p(maxf.data_ptr()), None)
    assert st == capi.EPI_OK, "epi_scan_block_noalloc returned %d" % st
    n = int(nhits.item())
    rows = hits[:min(n, cap)].cpu().numpy().copy().view(capi.HIT_DTYPE).reshape(-1)
    return rows, n, maxf.cpu().numpy()


def _by_pair(h):
    return h[np.lexsort((h["snp2"], h["snp1"]))]


@pytest.mark.parametrize("test,safe", [("i", 0), ("f", 1)])
def test_noalloc_matches_epi_scan(test, safe):
    torch = pytest.importorskip("torch")
    nid, sizes = 600, (180, 140)
    nsnp = sum(sizes)
    codes = synth.genotype_codes(nid, nsnp, seed=41)
    gp = synth.pack(codes)
    phen = synth.phenotype(nid, seed=42, miss=0.03)
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    t2 = synth.f_threshold(4, nid - 9, 1e-2)
    block = (sizes[0], sizes[1], 0, sizes[0])  # second chromosome x first
    opts = capi.default_opts(test=test, safe=safe, t1=t1, t2=t2, form=capi.FORM_POPC)

    with capi.Context(0) as ctx:
        ctx.load_packed(gp, nid)
        ctx.set_phenotype(phen, safe=safe)
        ref, ntot, ex = ctx.scan([block], opts)
        dump = ctx.scan_dump(block, opts)
    assert ntot > 20

    gp_dev = torch.from_numpy(np.ascontiguousarray(gp)).cuda()
    phen_dev = torch.from_numpy(np.ascontiguousarray(phen)).cuda()
    F_all = dump["F"].astype(np.float64)
    F2_all = dump["F2"].astype(np.float64)
    near = parity.near_threshold({"F": F_all, "F2": F2_all, "df1": dump["df1"]}, block, t1, t2, test, TOL_SET)
    for call in range(2):
        got, n, maxf = _noalloc(torch, gp_dev, nid, nsnp, phen_dev, block, opts, cap=4096)
        assert n == len(got) <= 4096
        ok, msg = parity.compare_hit_lists(_by_pair(got), _by_pair(ref), near)
        assert ok, "call %d: %s" % (call + 1, msg)
        a, b = _by_pair(got), _by_pair(ref)
        common = np.intersect1d(a["snp1"].astype(np.int64) * nsnp + a["snp2"],
                                b["snp1"].astype(np.int64) * nsnp + b["snp2"])
        ka = np.isin(a["snp1"].astype(np.int64) * nsnp + a["snp2"], common)
        kb = np.isin(b["snp1"].astype(np.int64) * nsnp + b["snp2"], common)
        assert np.array_equal(a["df1"][ka], b["df1"][kb]) and np.array_equal(a["df2"][ka], b["df2"][kb])
        assert parity.f_excess(a["F"][ka], b["F"][kb], b["df1"][kb], b["df2"][kb], F_TOL).max() <= 1.0
        if test == "i":
            assert parity.f_excess(a["F2"][ka], b["F2"][kb], b["df1"][kb], b["df2"][kb], F_TOL).max() <= 1.0
        assert abs(maxf[0] - ex["max_f"][0]) <= F_TOL * max(1.0, abs(ex["max_f"][0]))


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
