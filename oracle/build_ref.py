"""Build oracle A from the reference's own sources -- TEST INFRASTRUCTURE.

Reads src/EpiOpenCL.c of the reference tree (read-only; --reference or the EPIGPU_REFERENCE
environment variable), decodes
the C string literals that hold the OpenCL pair kernels

    kernelfull      src/EpiOpenCL.c:45-264   (8 df)
    kernelint       src/EpiOpenCL.c:276-504  (8 df + 4 df)
    kernelfullsafe  src/EpiOpenCL.c:507-726  (8 df, safe mode)
    kernelintsafe   src/EpiOpenCL.c:738-963  (8 df + 4 df, safe mode)

and compiles each one unmodified as C99 behind ref_prelude.h, renaming its entry point
`square` to `ref_<name>`. Linked with the NDRange emulator (ndrange_emu.c) they form
oracle/_ref/libepiref.so. The decoded kernel text only lives in a temporary directory;
the only output is the shared library under oracle/_ref/ (git-ignored, never committed).

Usage: python oracle/build_ref.py --reference DIR   (or EPIGPU_REFERENCE=DIR)
"""
import argparse
import os
import pathlib
import shutil
import subprocess
import sys
import tempfile

HERE = pathlib.Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
KERNELS = ("kernelfull", "kernelint", "kernelfullsafe", "kernelintsafe")


def extract_string(src: str, name: str) -> str:
    """Concatenate the adjacent string literals of `char *name = "..." "..." ;`.

    Handles backslash-newline continuations, // and /* */ comments between the
    literals, and the escapes the file uses (\\n, \\t, \\\\, \\")."""
    key = "char *%s =" % name
    pos = src.find(key)
    if pos < 0:
        raise ValueError("kernel string %s not found" % name)
    i = pos + len(key)
    out = []
    n = len(src)
    while i < n:
        c = src[i]
        if c == ";":
            return "".join(out)
        if c in " \t\r\n":
            i += 1
        elif c == "\\" and i + 1 < n and src[i + 1] in "\r\n":
            i += 1
        elif src.startswith("//", i):
            j = src.find("\n", i)
            i = n if j < 0 else j + 1
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            i = n if j < 0 else j + 2
        elif c == '"':
            i += 1
            while src[i] != '"':
                if src[i] == "\\":
                    e = src[i + 1]
                    out.append({"n": "\n", "t": "\t", "\\": "\\", '"': '"', "'": "'"}[e])
                    i += 2
                else:
                    out.append(src[i])
                    i += 1
            i += 1
        else:
            raise ValueError("unexpected character %r at offset %d in %s" % (c, i, name))
    raise ValueError("unterminated kernel string %s" % name)


def build(reference: pathlib.Path, out_dir: pathlib.Path = OUT_DIR, quiet: bool = False) -> pathlib.Path:
    src_file = reference / "src" / "EpiOpenCL.c"
    src = src_file.read_text(encoding="latin-1")
    out_dir.mkdir(parents=True, exist_ok=True)
    lib = out_dir / "libepiref.so"
    cc = shutil.which("gcc") or "gcc"  # the system gcc ships libgomp
    # float semantics: no contraction into FMA, no fast-math (IEEE single like the CL spec)
    cflags = ["-std=gnu99", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-w"]
    with tempfile.TemporaryDirectory(prefix="epiref_") as tmp:
        tmp = pathlib.Path(tmp)
        objs = []
        for name in KERNELS:
            text = extract_string(src, name)
            cl = tmp / (name + ".cl.c")
            cl.write_text(text)
            obj = tmp / (name + ".o")
            cmd = [cc, *cflags, "-include", str(HERE / "ref_prelude.h"),
                   "-Dsquare=ref_" + name, "-c", str(cl), "-o", str(obj)]
            subprocess.run(cmd, check=True)
            objs.append(str(obj))
        emu = tmp / "ndrange_emu.o"
        subprocess.run([cc, *cflags, "-fopenmp", "-I", str(HERE), "-c",
                        str(HERE / "ndrange_emu.c"), "-o", str(emu)], check=True)
        tmp_lib = tmp / "libepiref.so"
        subprocess.run([cc, "-shared", "-fopenmp", "-o", str(tmp_lib), str(emu), *objs, "-lm"],
                       check=True)
        shutil.copy2(tmp_lib, lib)
    if not quiet:
        print("built", lib)
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("EPIGPU_REFERENCE"))
    args = ap.parse_args()
    if not args.reference:
        ap.error("give the reference tree: --reference DIR or EPIGPU_REFERENCE=DIR")
    ref = pathlib.Path(args.reference)
    if not (ref / "src" / "EpiOpenCL.c").exists():
        print("reference sources not found at", ref, file=sys.stderr)
        sys.exit(1)
    build(ref)


if __name__ == "__main__":
    main()
