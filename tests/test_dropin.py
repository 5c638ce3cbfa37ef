"""The drop-in recipe for the reference's own build: epiGPU's
src/main.c, src/readplink.c and src/timing.c, compiled unmodified, with src/EpiOpenCL.c
replaced by epigpu_b200's perform_scan (epigpu_b200/host/scan_driver.c, the reference's
signature and globals, src/epiopencl.h:9-21) and -lOpenCL by libepigpu.so. The recipe is the
`refmain` target of oracle/Makefile, which writes oracle/_ref/epiGPU_refmain.

CPU: the recipe builds from the reference tree, and the binary runs the reference's own CLI
paths that need no GPU (usage text, argument checks, a clean "no suitable GPU" exit).
GPU: its `-A` results file is byte-identical to epigpu_b200's own epiGPU program on the same
data and options, with and without the reference's permutation (-p), 8 df and 4 df."""
import os
import pathlib
import subprocess

import pytest

from epigpu_b200 import epigpu_file, synth

ROOT = pathlib.Path(__file__).resolve().parents[1]
REFMAIN = ROOT / "oracle" / "_ref" / "epiGPU_refmain"
CLI = ROOT / "epigpu_b200" / "bin" / "epiGPU"
REFERENCE = os.environ.get("EPIGPU_REFERENCE", "")


def _gpu_present():
    try:
        from epigpu_b200 import capi
        with capi.Context(0):
            return True
    except Exception:
        return False


@pytest.mark.skipif(not REFMAIN.exists() and not REFERENCE, reason="oracle/_ref/epiGPU_refmain not built")
def test_recipe_links_reference_sources_to_the_library():
    if REFERENCE and (pathlib.Path(REFERENCE) / "src" / "main.c").exists():
        r = subprocess.run(["make", "-C", str(ROOT / "oracle"), "refmain", "REFERENCE=" + REFERENCE],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
    syms = subprocess.run(["nm", str(REFMAIN)], capture_output=True, text=True).stdout
    defined = {ln.split()[-1] for ln in syms.splitlines() if len(ln.split()) == 3 and ln.split()[1] in "TtBbDdCc"}
    # the reference's CLI and loader, epigpu_b200's scan driver; no OpenCL left
    for name in ("main", "analysismodecl", "readpackedbinary", "permute", "perform_scan", "resume_point",
                 "UFORM", "UNPERM", "UREFRESUME"):
        assert name in defined, name
    assert "clBuildProgram" not in syms
    assert "epi_scan" in syms  # resolved from libepigpu.so
    libs = subprocess.run(["ldd", str(REFMAIN)], capture_output=True, text=True).stdout
    assert "libepigpu.so" in libs and "OpenCL" not in libs


@pytest.mark.skipif(not REFMAIN.exists(), reason="oracle/_ref/epiGPU_refmain not built")
def test_reference_cli_paths_without_gpu(tmp_path):
    r = subprocess.run([str(REFMAIN)], capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert r.returncode == 1 and "ANALYSIS MODE" in r.stdout
    r = subprocess.run([str(REFMAIN), "-A", "x.epigpu", "out.txt", "-i", "20"], capture_output=True, text=True,
                       timeout=60, cwd=tmp_path)
    assert r.returncode != 0  # -i must be a multiple of 16 (src/main.c:123-129)
    if not _gpu_present():
        codes = synth.genotype_codes(100, 30, seed=1)
        d = epigpu_file.make(synth.pack(codes), 100, synth.phenotype(100, seed=2), [30])
        epigpu_file.write(tmp_path / "d.epigpu", d)
        r = subprocess.run([str(REFMAIN), "-A", "d.epigpu", "out.txt"], capture_output=True, text=True,
                           timeout=60, cwd=tmp_path)
        assert r.returncode == 1 and "no suitable GPU" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [["-t", "f"], ["-t", "i"], ["-t", "i", "-p", "3"], ["-t", "i", "-s", "1"]],
                         ids=["full", "int", "int_perm3", "int_safe"])
def test_dropin_results_match_own_cli(tmp_path, extra):
    assert REFMAIN.exists(), "oracle/_ref/epiGPU_refmain not built"
    nid, sizes = 400, (120, 90, 150)
    codes = synth.genotype_codes(nid, sum(sizes), seed=7)
    phen = synth.phenotype(nid, seed=8)
    d = epigpu_file.make(synth.pack(codes), nid, phen, list(sizes))
    epigpu_file.write(tmp_path / "data.epigpu", d)
    t1 = synth.f_threshold(8, nid - 9, 1e-2)
    t2 = synth.f_threshold(4, nid - 9, 1e-2)
    opts = ["-F", "%.6f" % t1, "-I", "%.6f" % t2, "-i", "32", *extra]
    outs = {}
    for name, exe in (("ref", REFMAIN), ("own", CLI)):
        run_dir = tmp_path / name
        run_dir.mkdir()
        (run_dir / "data.epigpu").symlink_to(tmp_path / "data.epigpu")
        r = subprocess.run([str(exe), "-A", "data.epigpu", "res.txt", *opts], capture_output=True, text=True,
                           timeout=300, cwd=run_dir)
        assert r.returncode == 0, name + ": " + r.stdout + r.stderr
        outs[name] = (run_dir / "res.txt").read_text()
    assert outs["ref"] == outs["own"]
    rows = [ln for ln in outs["ref"].splitlines() if ln and ln[0].isdigit()]
    assert len(rows) > 20
    if "-p" in extra:  # the reference's permute writes the permuted phenotypes (src/main.c:349-356)
        assert (tmp_path / "ref" / "perm3.txt").exists()
