"""Data mode of the host program: epiGPU -Dr (PLINK .ped/.map -> .epigpu) and -De (the
inverse), against the reference's own data-mode functions (src/readplink.c, built
unmodified into oracle/_ref/plinkref). On space-delimited PLINK files the .epigpu file and
the extracted text must be byte-for-byte the reference's; tab-delimited files (which the
reference's allele scan misreads) must give the same file as their space-delimited twin."""
import subprocess

import numpy as np
import pytest

from epigpu_b200 import epigpu_file

ROOT = __import__("pathlib").Path(__file__).resolve().parents[1]
CLI = ROOT / "epigpu_b200" / "bin" / "epiGPU"
REF = ROOT / "oracle" / "_ref" / "plinkref"

needs_cli = pytest.mark.skipif(not CLI.exists(), reason="host program not built")
needs_ref = pytest.mark.skipif(not REF.exists(), reason="reference data-mode oracle not built")


def write_plink(d, nid, nsnp, seed, sep=" ", binary=False, third_allele=False, interleave=False,
                half_missing=True):
    """A seeded PLINK fileset: per SNP two of A/C/G/T; genotypes drawn among both homozygotes,
    both heterozygote orders, missing (0 0) and half-missing (X 0); every SNP has a
    homozygote (individual 0), as the reference requires, and a heterozygote (individual 1)."""
    rng = np.random.default_rng(seed)
    letters = "ACGT"
    alle = [rng.choice(4, 3, replace=False) for _ in range(nsnp)]
    p = [0.3, 0.15, 0.15, 0.25, 0.1, 0.05] if half_missing else [0.3, 0.15, 0.15, 0.3, 0.1, 0.0]
    G = rng.choice(6, (nid, nsnp), p=p)
    G[0, :] = 0
    G[1, :] = 1
    if third_allele:
        G[rng.integers(1, nid, 3), 1] = 6  # homozygote of a third allele at SNP 1
    lines = []
    for i in range(nid):
        phen = str(1 + int(rng.integers(0, 2))) if binary else ("-9" if i % 7 == 3 else "%.6f" % rng.standard_normal())
        f = ["F%d" % (i // 3), "ind%d" % i, "0", "pat%d" % i, str(1 + i % 2), phen]
        for j in range(nsnp):
            a, b, c = (letters[k] for k in alle[j])
            f += {0: [a, a], 1: [a, b], 2: [b, a], 3: [b, b], 4: ["0", "0"], 5: [a, "0"], 6: [c, c]}[int(G[i, j])]
        lines.append(sep.join(f))
    (d / "x.ped").write_text("\n".join(lines) + "\n")
    chrs = sorted(rng.integers(1, 5, nsnp).tolist())
    if interleave:
        chrs[len(chrs) // 2] = chrs[0]  # a chromosome name that comes back later in the map
    names = ["chr%d" % c for c in chrs]
    (d / "x.map").write_text("".join("%s rs%d %.4f %d\n" % (n, 1000 + j, 0.01 * j, 5000 + 37 * j)
                                     for j, n in enumerate(names)))
    return d / "x.ped", d / "x.map"


def run(*args, ok=True):
    r = subprocess.run([str(a) for a in args], capture_output=True, text=True, timeout=120)
    if ok:
        assert r.returncode == 0, r.stdout + r.stderr
    return r


@needs_cli
@needs_ref
@pytest.mark.parametrize("nid,nsnp,kw", [
    (37, 23, {}),
    (64, 40, {"binary": True}),
    (10, 10, {}),
    (129, 31, {"third_allele": True}),
    (50, 60, {"interleave": True}),
], ids=["tail-word-37", "binary-64", "minimal-10", "third-allele", "interleaved-chr"])
def test_read_plink_matches_reference(tmp_path, nid, nsnp, kw):
    ped, mp = write_plink(tmp_path, nid, nsnp, seed=nid + nsnp, **kw)
    run(CLI, "-Dr", ped, mp, tmp_path / "ours.epigpu")
    run(REF, "write", ped, mp, tmp_path / "ref.epigpu")
    ours, ref = (tmp_path / "ours.epigpu").read_bytes(), (tmp_path / "ref.epigpu").read_bytes()
    assert ours == ref, "the .epigpu file differs from the reference's"
    d = epigpu_file.read(tmp_path / "ours.epigpu")
    assert (d.nid, d.nsnp) == (nid, nsnp)

    # extraction, both ways from the same file
    run(CLI, "-De", tmp_path / "o.ped", tmp_path / "o.map", tmp_path / "ours.epigpu")
    run(REF, "extract", tmp_path / "ours.epigpu", tmp_path / "r.ped", tmp_path / "r.map")
    assert (tmp_path / "o.ped").read_bytes() == (tmp_path / "r.ped").read_bytes()
    assert (tmp_path / "o.map").read_bytes() == (tmp_path / "r.map").read_bytes()


@needs_cli
def test_round_trip_keeps_genotypes(tmp_path):
    """-Dr, -De, -Dr gives the same genotype words. The format only carries that when every
    SNP has a true heterozygote (which sets both allele names) and no half-missing call
    (which the reference codes as a heterozygote and takes '0' as an allele name)."""
    ped, mp = write_plink(tmp_path, 80, 33, seed=3, half_missing=False)
    run(CLI, "-Dr", ped, mp, tmp_path / "a.epigpu")
    run(CLI, "-De", tmp_path / "b.ped", tmp_path / "b.map", tmp_path / "a.epigpu")
    run(CLI, "-Dr", tmp_path / "b.ped", tmp_path / "b.map", tmp_path / "b.epigpu")
    a, b = epigpu_file.read(tmp_path / "a.epigpu"), epigpu_file.read(tmp_path / "b.epigpu")
    assert np.array_equal(a.gpack, b.gpack)
    assert np.array_equal(a.genmap["allelename"], b.genmap["allelename"])
    assert np.array_equal(a.chrom, b.chrom)
    np.testing.assert_allclose(a.ped["phen"], b.ped["phen"], rtol=1e-6)


@needs_cli
def test_tab_delimited_reads_like_space_delimited(tmp_path):
    sp, tb = tmp_path / "sp", tmp_path / "tb"
    sp.mkdir()
    tb.mkdir()
    ped1, map1 = write_plink(sp, 45, 19, seed=9)
    ped2, map2 = write_plink(tb, 45, 19, seed=9, sep="\t")
    run(CLI, "-Dr", ped1, map1, tmp_path / "sp.epigpu")
    run(CLI, "-Dr", ped2, map2, tmp_path / "tb.epigpu")
    assert (tmp_path / "sp.epigpu").read_bytes() == (tmp_path / "tb.epigpu").read_bytes()


@needs_cli
def test_data_mode_errors(tmp_path):
    ped, mp = write_plink(tmp_path, 20, 12, seed=1)
    text = ped.read_text().splitlines()
    rag = tmp_path / "rag.ped"
    rag.write_text("\n".join(text[:5] + [text[5] + " A A"] + text[6:]) + "\n")
    r = run(CLI, "-Dr", rag, mp, tmp_path / "o.epigpu", ok=False)
    assert r.returncode != 0 and "Ragged" in r.stdout
    long = tmp_path / "long.ped"
    fields = text[0].split(" ")
    fields[1] = "x" * 40
    long.write_text("\n".join([" ".join(fields)] + text[1:]) + "\n")
    r = run(CLI, "-Dr", long, mp, tmp_path / "o.epigpu", ok=False)
    assert r.returncode != 0 and "longer than 29" in r.stdout
    r = run(CLI, "-Drm", ped, mp, tmp_path / "o.epigpu", ok=False)
    assert r.returncode != 0 and "not part of" in r.stdout
    r = run(CLI, "-Dr", ped, mp, ok=False)
    assert r.returncode != 0


GOLDEN = ROOT / "tests" / "golden"
PLINK_CASES = __import__("json").loads((GOLDEN / "plink_cases.json").read_text())


@needs_cli
@pytest.mark.parametrize("case", PLINK_CASES, ids=[c["name"] for c in PLINK_CASES])
def test_read_plink_matches_golden(tmp_path, case):
    """Against the reference's recorded outputs (tests/golden/, written by its own readplink.c
    functions): no reference tree needed."""
    import hashlib
    ped, mp = write_plink(tmp_path, case["nid"], case["nsnp"], seed=case["seed"], **case["kw"])
    assert hashlib.sha256(ped.read_bytes()).hexdigest() == case["ped_sha256"], "fileset generator changed"
    assert hashlib.sha256(mp.read_bytes()).hexdigest() == case["map_sha256"], "fileset generator changed"
    run(CLI, "-Dr", ped, mp, tmp_path / "ours.epigpu")
    assert (tmp_path / "ours.epigpu").read_bytes() == (GOLDEN / ("%s.epigpu" % case["name"])).read_bytes()
    run(CLI, "-De", tmp_path / "o.ped", tmp_path / "o.map", GOLDEN / ("%s.epigpu" % case["name"]))
    assert (tmp_path / "o.ped").read_bytes() == (GOLDEN / ("%s.ped" % case["name"])).read_bytes()
    assert (tmp_path / "o.map").read_bytes() == (GOLDEN / ("%s.map" % case["name"])).read_bytes()
