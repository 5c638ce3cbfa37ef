"""The host program end to end on the GPU: `epiGPU -A` on a .epigpu file against the results
file the reference would write (rows from oracle A, the reference's kernels, block by block),
plus checkpoint/resume from a results file cut after a complete block
(src/EpiOpenCL.c:1187-1274, :1442-1470)."""
import pathlib
import subprocess

import numpy as np
import pytest

import oracles
import parity
from epigpu_b200 import epigpu_file, synth

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parents[1]
CLI = ROOT / "epigpu_b200" / "bin" / "epiGPU"


def parse_results(path):
    lines = pathlib.Path(path).read_text().splitlines()
    header = lines[:8]
    blocks = []
    i = 8
    while i < len(lines):
        parts = lines[i].split()
        assert parts[0] == "#", lines[i]
        c1, c2, n = int(parts[1]), int(parts[3]), int(parts[5])
        rows = [ln.split("\t") for ln in lines[i + 1:i + 1 + n]]
        blocks.append((c1, c2, rows))
        i += 1 + n
    return header, blocks


def make_data(tmp_path, nid=300, sizes=(90, 140, 60), seed=5):
    codes = synth.genotype_codes(nid, sum(sizes), seed=seed)
    phen = synth.phenotype(nid, seed=seed + 1)
    d = epigpu_file.make(synth.pack(codes), nid, phen, list(sizes))
    path = tmp_path / "data.epigpu"
    epigpu_file.write(path, d)
    return path, d, codes, phen


@pytest.mark.parametrize("test,form", [("f", "p"), ("i", "p"), ("i", "t")])
def test_results_file_matches_reference(tmp_path, test, form):
    path, d, codes, phen = make_data(tmp_path)
    out = tmp_path / "res.txt"
    t1 = synth.f_threshold(8, d.nid - 9, 1e-2)
    t2 = synth.f_threshold(4, d.nid - 9, 1e-2)
    r = subprocess.run([str(CLI), "-A", str(path), str(out), "-t", test, "-F", "%.6f" % t1, "-I", "%.6f" % t2,
                        "-i", "32", "-g", form], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    header, blocks = parse_results(out)
    assert header[0] == "Datafile: data.epigpu "
    assert header[1] == "Number of individuals: %d" % d.nid
    assert header[5] == ("Test: full" if test == "f" else "Test: interactions + full")
    want_blocks = [(i, j) for i in range(d.nchr) for j in range(i + 1)]
    assert [(b[0], b[1]) for b in blocks] == want_blocks
    t1f, t2f = float(np.float32(t1)), float(np.float32(t2))
    for (c1, c2, rows), blk in zip(blocks, d.blocks()):
        got = np.array([(int(x[0]) - 1, int(x[3]) - 1) for x in rows], dtype=[("snp1", "i4"), ("snp2", "i4")])
        hb, tb, pb = oracles.oracle_scan_block(codes, phen, blk, test=test, chunk=32, t1=t1f, t2=t2f, per_pair=True)
        excl = parity.near_threshold(pb, blk, t1f, t2f, test, 1e-4)
        ok, msg = parity.compare_hit_lists(got, hb, excl)
        assert ok, "block %d x %d: %s" % (c1, c2, msg)
        if oracles.have_ref():
            ha, _ = oracles.ref_scan_block(d.gpack, d.nid, phen, blk, test=test, chunk=32, t1=t1f, t2=t2f,
                                           nthreads=8)
            ok, msg = parity.compare_hit_lists(got, ha, excl)
            assert ok, "block %d x %d vs reference: %s" % (c1, c2, msg)
        for x in rows:
            s1, s2 = int(x[0]) - 1, int(x[3]) - 1
            assert x[1] == "rs%d" % (s1 + 1) and x[4] == "rs%d" % (s2 + 1)
            assert x[2] == str(c1 + 1) and x[5] == str(c2 + 1)
            gx, gy = s1 - blk[0], s2 - blk[2]
            assert int(x[6]) == pb["df1"][gx, gy] and int(x[7]) == pb["df2"][gx, gy]
            assert abs(float(x[8]) - pb["F"][gx, gy]) <= 1e-5 * max(1.0, abs(pb["F"][gx, gy])) + 5e-7


def test_resume_after_interruption(tmp_path):
    path, d, codes, phen = make_data(tmp_path, sizes=(50, 70, 40, 30))
    full = tmp_path / "full.txt"
    args = ["-t", "i", "-F", "3", "-I", "4"]
    r = subprocess.run([str(CLI), "-A", str(path), str(full), *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    text = full.read_text().splitlines(keepends=True)
    # cut the file after the third block and in the middle of the fourth
    header, blocks = parse_results(full)
    keep = 8 + sum(1 + len(b[2]) for b in blocks[:3])
    part = tmp_path / "part.txt"
    part.write_text("".join(text[:keep + 2]))
    r = subprocess.run([str(CLI), "-A", str(path), str(part), *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    assert "Resuming from" in r.stdout
    # the partial block is dropped and rescanned: the resumed file is the uninterrupted one
    assert part.read_text() == full.read_text()
    r = subprocess.run([str(CLI), "-A", str(path), str(full), *args], capture_output=True, text=True, timeout=300)
    assert "Scan already completed" in r.stdout


def test_resume_reference_rule(tmp_path):
    """Interrupted after block (2, 0): the default resume scans (2, 1), (2, 2) and every block of
    chromosome 3; -R 1 restarts chromosome 3 at column 1 as the reference's loop does
    (src/EpiOpenCL.c:1540) and so leaves out block (3, 0)."""
    path, d, codes, phen = make_data(tmp_path, sizes=(50, 70, 40, 30))
    full = tmp_path / "full.txt"
    args = ["-t", "f", "-F", "3"]
    r = subprocess.run([str(CLI), "-A", str(path), str(full), *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    header, blocks = parse_results(full)
    assert [(b[0], b[1]) for b in blocks][3] == (2, 0)
    keep = 8 + sum(1 + len(b[2]) for b in blocks[:4])
    text = full.read_text().splitlines(keepends=True)
    for flag, want in (("0", blocks), ("1", [b for b in blocks if (b[0], b[1]) != (3, 0)])):
        part = tmp_path / ("part%s.txt" % flag)
        part.write_text("".join(text[:keep]))
        r = subprocess.run([str(CLI), "-A", str(path), str(part), *args, "-R", flag], capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stdout
        _, got = parse_results(part)
        assert got == want, "-R %s" % flag



def test_plink_fileset_to_scan(tmp_path):
    """PLINK text in, results out: epiGPU -Dr turns a .ped/.map fileset into a .epigpu file
    and epiGPU -A scans it (tensor form); the hits match the FP64 oracle run on the genotype
    codes and phenotypes the file holds."""
    import test_datamode
    ped, mp = test_datamode.write_plink(tmp_path, 300, 150, seed=21)
    path = tmp_path / "plink.epigpu"
    r = subprocess.run([str(CLI), "-Dr", str(ped), str(mp), str(path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    d = epigpu_file.read(path)
    codes = oracles.oracle_unpack(d.gpack, d.nid)
    phen = d.ped["phen"].astype(np.float32)
    out = tmp_path / "res.txt"
    t1 = float(np.float32(synth.f_threshold(8, d.nid - 9, 5e-2)))
    t2 = float(np.float32(synth.f_threshold(4, d.nid - 9, 5e-2)))
    r = subprocess.run([str(CLI), "-A", str(path), str(out), "-t", "i", "-F", "%.6f" % t1, "-I", "%.6f" % t2,
                        "-g", "t"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    header, blocks = parse_results(out)
    assert len(blocks) == d.nchr * (d.nchr + 1) // 2
    total = 0
    for (c1, c2, rows), blk in zip(blocks, d.blocks()):
        got = np.array([(int(x[0]) - 1, int(x[3]) - 1) for x in rows], dtype=[("snp1", "i4"), ("snp2", "i4")])
        hb, tb, pb = oracles.oracle_scan_block(codes, phen, blk, test="i", t1=t1, t2=t2, per_pair=True)
        excl = parity.near_threshold(pb, blk, t1, t2, "i", 1e-4)
        ok, msg = parity.compare_hit_lists(got, hb, excl)
        assert ok, "block %d x %d: %s" % (c1, c2, msg)
        total += len(rows)
    assert total > 0


def test_permutation_threshold(tmp_path):
    """-N n scans n permuted phenotypes (the -p rule, p = 1..n) in the same launches: the
    results file is the one a plain run writes, and <output>.perm holds each permutation's
    largest F / Fint over every pair, which must match the FP64 oracle's maximum for that
    permuted phenotype, with the family-wise thresholds and p-value computed from them."""
    path, d, codes, phen = make_data(tmp_path, nid=300, sizes=(70, 50), seed=8)
    K = 20
    plain, perm = tmp_path / "plain.txt", tmp_path / "perm.txt"
    args = ["-t", "i", "-F", "5.0", "-I", "6.0", "-g", "t"]
    for out, extra in ((plain, []), (perm, ["-N", str(K)])):
        r = subprocess.run([str(CLI), "-A", str(path), str(out), *args, *extra], capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
    assert plain.read_text() == perm.read_text()
    lines = (tmp_path / "perm.txt.perm").read_text().splitlines()
    head = dict(ln.split(": ", 1) for ln in lines if ": " in ln)
    table = lines[lines.index("Perm\tmaxF\tmaxFint") + 1:]
    assert len(table) == K
    got = np.array([[float(x) for x in ln.split("\t")[1:]] for ln in table])

    def max_stats(y):
        mf = mf2 = -np.inf
        for blk in d.blocks():
            _, _, pb = oracles.oracle_scan_block(codes, y, blk, test="i", t1=1e30, t2=1e30, per_pair=True)
            s1, m1, s2, m2 = blk
            gx, gy = np.meshgrid(np.arange(m1), np.arange(m2), indexing="ij")
            ok = (gx + s1 > gy + s2) & np.isfinite(pb["F"]) & (pb["df1"] > 0)
            mf = max(mf, pb["F"][ok].max())
            mf2 = max(mf2, pb["F2"][ok & np.isfinite(pb["F2"])].max())
        return mf, mf2

    obs = max_stats(phen)
    assert abs(float(head["Observed largest F"]) - obs[0]) <= 1e-5 * obs[0] + 1e-6
    want = np.array([max_stats(oracles.oracle_permute(phen, p)) for p in range(1, K + 1)])
    assert np.all(np.abs(got - want) <= 1e-5 * np.abs(want) + 1e-6), np.abs(got - want).max()
    srt = np.sort(got[:, 0])
    assert abs(float(head["Family-wise 5% threshold for F"]) - srt[int(np.ceil(0.95 * K)) - 1]) <= 1e-5 * srt[-1]
    pval = (1 + np.sum(got[:, 0] >= float(head["Observed largest F"]))) / (K + 1)
    assert abs(float(head["Family-wise p-value of the observed largest F"]) - pval) < 1e-6
