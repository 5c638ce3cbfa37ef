"""Golden fixtures (tests/golden/): hit lists of the reference's own pair kernels on seeded
inputs, recorded by tests/golden/make_golden.py. They pin the FP64 oracle (CPU) and the CUDA
forms (GPU) to the reference's outputs without needing the reference tree.

Bars: the same pairs in the same order (the reference's output order) except pairs whose
FP64 F or F2 lies within 1e-3 relative of a threshold; df exact; the reference's float32 F
within 5e-5 x kappa of FP64 (its own rounding at these N)."""
import hashlib
import json
import pathlib

import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import capi, synth

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
CASES = json.loads((GOLDEN / "cases.json").read_text())
IDS = [c["name"] for c in CASES]
TOL_SET = 1e-3
F32_TOL = 5e-5


def _inputs(case):
    codes = synth.genotype_codes(case["nid"], case["nsnp"], seed=case["seed"], miss=case["miss_g"])
    phen = synth.phenotype(case["nid"], seed=case["seed"] + 1, miss=case["miss_p"])
    return codes, synth.pack(codes), phen


def _golden(case):
    z = np.load(GOLDEN / ("%s.npz" % case["name"]))
    out = np.zeros(len(z["snp1"]), dtype=capi.HIT_DTYPE)
    for k in ("snp1", "snp2", "df1", "df2", "F", "F2"):
        out[k] = z[k]
    return out


def _compare(got, gold, pb, case):
    blk = tuple(case["block"])
    excl = parity.near_threshold(pb, blk, case["t1"], case["t2"], case["test"], TOL_SET)
    ok, msg = parity.compare_hit_lists(got, gold, excl)
    assert ok, msg
    where = {k: i for i, k in enumerate(parity.pair_key(gold))}
    idx = np.array([(i, where[k]) for i, k in enumerate(parity.pair_key(got)) if k in where])
    gi, ri = idx.T
    assert np.array_equal(got["df1"][gi], gold["df1"][ri]) and np.array_equal(got["df2"][gi], gold["df2"][ri])
    for f in ("F", "F2") if case["test"] == "i" else ("F",):
        e = parity.f_excess(gold[f][ri], got[f][gi], got["df1"][gi], got["df2"][gi], F32_TOL)
        assert e.max() <= 1.0, "%s: %.3g x bound" % (f, e.max())


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_golden_inputs_regenerate(case):
    _, gp, phen = _inputs(case)
    assert hashlib.sha256(np.ascontiguousarray(gp).tobytes()).hexdigest() == case["gpack_sha256"]
    assert hashlib.sha256(np.ascontiguousarray(phen).tobytes()).hexdigest() == case["phen_sha256"]


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_fp64_oracle_matches_golden(case):
    codes, gp, phen = _inputs(case)
    hb, tb, pb = oracles.oracle_scan_block(codes, phen, tuple(case["block"]), test=case["test"], safe=case["safe"],
                                           chunk=case["chunk"], t1=case["t1"], t2=case["t2"], per_pair=True)
    _compare(hb, _golden(case), pb, case)


@pytest.mark.gpu
@pytest.mark.parametrize("form", [capi.FORM_POPC, capi.FORM_TENSOR], ids=["popc", "tensor"])
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_cuda_forms_match_golden(gpu_ctx, case, form):
    codes, gp, phen = _inputs(case)
    gpu_ctx.load_packed(gp, case["nid"])
    gpu_ctx.set_phenotype(phen, safe=case["safe"])
    opts = capi.default_opts(test=case["test"], safe=case["safe"], chunk=case["chunk"], t1=case["t1"],
                             t2=case["t2"], form=form)
    got, total, _ = gpu_ctx.scan([tuple(case["block"])], opts)
    _, _, pb = oracles.oracle_scan_block(codes, phen, tuple(case["block"]), test=case["test"], safe=case["safe"],
                                         chunk=case["chunk"], t1=case["t1"], t2=case["t2"], per_pair=True)
    _compare(got, _golden(case), pb, case)
