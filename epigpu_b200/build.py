"""Builds the native parts of epigpu_b200 in-tree.

  epigpu_b200/libepigpu.so   CUDA kernels + C ABI (nvcc, sm_100a only)
  epigpu_b200/bin/epiGPU     the C host program (CLI, .epigpu loader, results file)

Usage: python -m epigpu_b200.build [--no-cli] [-v]
"""
import argparse
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
INCLUDE = ROOT / "include"
LIB = PKG / "libepigpu.so"
CLI = PKG / "bin" / "epiGPU"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _gcc():
    return shutil.which("gcc") or "gcc"


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd))
    subprocess.run([str(c) for c in cmd], check=True)


def _stale(target: pathlib.Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_lib(verbose=False, ptxas_v=False, force=False):
    sources = sorted(CSRC.glob("*.cu"))
    deps = sources + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "epigpu.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in sources:
        obj = objdir / (src.stem + ".o")
        cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
        if ptxas_v:
            cmd[1:1] = ["-Xptxas", "-v"]
        _run(cmd, verbose)
        objs.append(obj)
    tmp = LIB.with_suffix(".so.tmp")
    _run([_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp,
          "-lcuda"], verbose)
    os.replace(tmp, LIB)
    return LIB


def build_cli(verbose=False, force=False):
    sources = sorted(HOST.glob("*.c"))
    if not sources:
        return None
    deps = sources + sorted(HOST.glob("*.h")) + [INCLUDE / "epigpu.h", LIB]
    if not force and not _stale(CLI, deps):
        return CLI
    CLI.parent.mkdir(exist_ok=True)
    _run([_gcc(), "-std=gnu99", "-O2", "-Wall", "-Wno-unused-result", "-I", INCLUDE, "-I", HOST,
          *sources, "-o", CLI, "-L", PKG, "-lepigpu", "-Wl,-rpath,$ORIGIN/..", "-lm"], verbose)
    return CLI


def build(verbose=False, cli=True, force=False):
    build_lib(verbose=verbose, force=force)
    if cli:
        build_cli(verbose=verbose, force=force)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--no-cli", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args()
    if args.ptxas_v:
        build_lib(verbose=True, ptxas_v=True, force=True)
    else:
        build(verbose=args.verbose, cli=not args.no_cli, force=args.force)
    print("built", LIB)


if __name__ == "__main__":
    sys.exit(main())
