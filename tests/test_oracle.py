"""CPU tests of the oracles: oracle B (FP64 restatement) pinned against oracle A (the
reference's own kernels built from its sources), plus the packing, file-format and
permutation rules. The committed golden fixtures (reference outputs) are checked in
test_golden.py."""
import numpy as np
import pytest

import oracles
from epigpu_b200 import synth

needs_ref = pytest.mark.skipif(not oracles.have_ref(), reason="oracle A not built (no reference tree)")


@pytest.mark.parametrize("nid", [1, 7, 16, 17, 31, 32, 500])
def test_pack_roundtrip_matches_reference_rule(nid):
    codes = synth.genotype_codes(nid, 23, seed=nid, miss=0.1)
    gp = synth.pack(codes)
    assert np.array_equal(gp, oracles.oracle_pack(codes))
    assert np.array_equal(synth.unpack(gp, nid), codes)
    assert np.array_equal(oracles.oracle_unpack(gp, nid), codes)


def test_tail_word_is_right_aligned():
    # readplink.c:1090-1098: the first leftover individual sits at bit 2*(remain-1)
    codes = np.zeros((1, 19), dtype=np.uint8)
    codes[0, 16] = 1
    codes[0, 18] = 2
    gp = synth.pack(codes).view(np.uint32)
    assert gp[0, 1] == (1 << 4) | 2


@needs_ref
@pytest.mark.parametrize("test,safe", [("f", 0), ("i", 0), ("f", 1), ("i", 1)])
def test_fp64_oracle_matches_reference_kernels(test, safe):
    nid, nsnp = 211, 150
    codes = synth.genotype_codes(nid, nsnp, seed=3, miss=0.03)
    gp = synth.pack(codes)
    phen = synth.phenotype(nid, seed=4, miss=0.05)
    blk = (0, nsnp, 0, nsnp)
    ha, ta, ca, _ = oracles.ref_scan_block(gp, nid, phen, blk, test=test, safe=safe, t1=-1e30, t2=-1e30,
                                           dump=True, nthreads=4)
    hb, tb, pb = oracles.oracle_scan_block(codes, phen, blk, test=test, safe=safe, t1=-1e30, t2=-1e30,
                                           per_pair=True)
    tri = np.tril(np.ones((nsnp, nsnp), bool), -1)
    assert np.array_equal(ca[tri], pb["counts"][tri])
    assert ta == tb
    assert np.array_equal(ha["snp1"], hb["snp1"]) and np.array_equal(ha["snp2"], hb["snp2"])
    assert np.array_equal(ha["df1"], hb["df1"]) and np.array_equal(ha["df2"], hb["df2"])
    # the reference's float32 F against FP64: the float32 envelope at this N
    assert oracles.rel_err(ha["F"], hb["F"]).max() < 2e-5


@needs_ref
def test_reference_order_is_slot_major():
    """perform_scan writes a block slot by slot (EpiOpenCL.c:1621)."""
    nid, nsnp = 64, 100
    codes = synth.genotype_codes(nid, nsnp, seed=8)
    gp = synth.pack(codes)
    phen = synth.phenotype(nid, seed=9)
    ha, _ = oracles.ref_scan_block(gp, nid, phen, (0, nsnp, 0, nsnp), t1=-1e30, chunk=32)
    s = (ha["snp1"] % 16) * 16 + ha["snp2"] % 16
    assert np.all(np.diff(s) >= 0)
    hs, _ = oracles.ref_scan_block(gp, nid, phen, (0, nsnp, 0, nsnp), t1=-1e30, chunk=32, nthreads=4)
    assert np.array_equal(ha, hs)


@needs_ref
def test_reference_off_diagonal_block():
    nid = 90
    codes = synth.genotype_codes(nid, 120, seed=12)
    gp = synth.pack(codes)
    phen = synth.phenotype(nid, seed=13)
    blk = (70, 50, 0, 70)
    ha, ta = oracles.ref_scan_block(gp, nid, phen, blk, test="i", t1=1.5, t2=1.5)
    hb, tb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=1.5, t2=1.5)
    assert ta == tb
    assert np.array_equal(ha["snp1"], hb["snp1"]) and np.array_equal(ha["snp2"], hb["snp2"])


def test_permutation_rule():
    phen = np.arange(50, dtype=np.float32)
    p = oracles.oracle_permute(phen, 7)
    assert sorted(p.tolist()) == phen.tolist()
    assert not np.array_equal(p, phen)
    assert np.array_equal(p, oracles.oracle_permute(phen, 7))
