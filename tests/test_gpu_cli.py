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

