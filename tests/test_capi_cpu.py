"""CPU tests of the boundary: the C-ABI library loads and exports what include/epigpu.h
declares, fails cleanly without a GPU, and the C host program's command line, .epigpu
reader and error paths behave like the reference's (src/main.c:58-188,
src/readplink.c:1183-1273). No GPU compute here."""
import ctypes
import pathlib
import re
import subprocess

import numpy as np
import pytest

from epigpu_b200 import capi, epigpu_file, synth

ROOT = pathlib.Path(__file__).resolve().parents[1]
CLI = ROOT / "epigpu_b200" / "bin" / "epiGPU"


def declared_functions():
    text = (ROOT / "include" / "epigpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(epi_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_functions()
    assert set(names) == set(capi.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(r"\bT %s$" % n, out, re.M), n


def test_struct_layouts_match_reference():
    # table (src/id4117.h:14-21) is 24 bytes; the options struct is fixed at 64
    assert ctypes.sizeof(capi.Hit) == 24
    assert ctypes.sizeof(capi.Block) == 16
    assert ctypes.sizeof(capi.ScanOpts) == 64
    assert epigpu_file.PED.itemsize == 128 and epigpu_file.MAP.itemsize == 88 and epigpu_file.CHROM.itemsize == 44


def test_defaults_are_the_reference_defaults():
    o = capi.default_opts()
    assert chr(o.test) == "f" and o.safe == 0 and o.chunk == 128
    assert abs(o.t1 - 6.5) < 1e-7 and abs(o.t2 - 10.5) < 1e-7


def test_strerror_and_open_without_gpu():
    lib = capi.load()
    for s in range(9):
        assert lib.epi_strerror(s)
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        with pytest.raises(capi.EpiError) as e:
            capi.Context(0)
        assert e.value.status == capi.EPI_E_NODEVICE


def test_permutation_matches_glibc_rule():
    import oracles
    phen = synth.phenotype(97, seed=3)
    for seed in (1, 2, 100):
        assert np.array_equal(capi.permute_phenotype(phen, seed), oracles.oracle_permute(phen, seed))


def _write(tmp_path, nid=50, sizes=(30, 20)):
    codes = synth.genotype_codes(nid, sum(sizes), seed=1)
    d = epigpu_file.make(synth.pack(codes), nid, synth.phenotype(nid, seed=2), list(sizes))
    path = tmp_path / "d.epigpu"
    epigpu_file.write(path, d)
    return path, d


def test_epigpu_file_roundtrip(tmp_path):
    path, d = _write(tmp_path)
    r = epigpu_file.read(path)
    assert r.nid == d.nid and r.nsnp == d.nsnp and r.nchr == 2
    assert np.array_equal(r.gpack, d.gpack)
    assert np.array_equal(r.ped["phen"], d.ped["phen"])
    assert r.blocks() == [(0, 30, 0, 30), (30, 20, 0, 30), (30, 20, 30, 20)]


def run_cli(*args, cwd=None):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=60)


@pytest.mark.skipif(not CLI.exists(), reason="host program not built")
def test_cli_argument_checks(tmp_path):
    path, _ = _write(tmp_path)
    out = tmp_path / "o.txt"
    cases = [
        (["-A", path], "Incorrect arguments"),
        (["-A", path, out, "-i", "20"], "Iteration size must be a multiple of 16"),
        (["-A", path, out, "-i", "x"], "numeric value for iteration size"),
        (["-A", path, out, "-t", "q"], "Test selection"),
        (["-A", path, out, "-F", "0"], "numeric F-test threshold"),
        (["-A", path, out, "-s", "2"], "Safe mode option"),
        (["-A", path, out, "-P", tmp_path / "missing.txt"], "Separate phenotype file does not exist"),
        (["-A", path, out, "-g", "z"], "GPU form"),
    ]
    for args, msg in cases:
        r = run_cli(*args)
        assert r.returncode == 1, args
        assert msg in r.stdout, (args, r.stdout)


@pytest.mark.skipif(not CLI.exists(), reason="host program not built")
def test_cli_rejects_bad_files(tmp_path):
    path, _ = _write(tmp_path)
    raw = path.read_bytes()
    bad = tmp_path / "bad.epigpu"
    bad.write_bytes(b"XXXXXX" + raw[6:])
    assert "Invalid input file" in run_cli("-A", bad, tmp_path / "o.txt").stdout
    bad.write_bytes(raw[:-10])
    r = run_cli("-A", bad, tmp_path / "o.txt")
    assert r.returncode == 1 and "truncated" in r.stdout
    r = run_cli("-A", tmp_path / "nope.epigpu", tmp_path / "o.txt")
    assert r.returncode == 1 and "No input file found" in r.stdout


@pytest.mark.skipif(not CLI.exists(), reason="host program not built")
def test_cli_rejects_binary_phenotype(tmp_path):
    nid = 40
    codes = synth.genotype_codes(nid, 10, seed=1)
    d = epigpu_file.make(synth.pack(codes), nid, np.where(np.arange(nid) % 2, 1.0, 2.0), [10])
    path = tmp_path / "b.epigpu"
    epigpu_file.write(path, d)
    r = run_cli("-A", path, tmp_path / "o.txt")
    assert r.returncode == 1 and "Binary phenotype" in r.stdout
