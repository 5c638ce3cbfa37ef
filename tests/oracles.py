"""ctypes wrappers of the two oracles (test infrastructure only).

  A  oracle/_ref/libepiref.so  the reference's own OpenCL kernels compiled as C,
                               driven like perform_scan (float32, reference hit order)
  B  oracle/liboracle.so       FP64 restatement of the same statistics
"""
import ctypes
import pathlib
import subprocess

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
ORACLE = ROOT / "oracle"
REF_LIB = ORACLE / "_ref" / "libepiref.so"
B_LIB = ORACLE / "liboracle.so"

REF_HIT = np.dtype([("snp1", "<i4"), ("snp2", "<i4"), ("df1", "<i4"), ("df2", "<i4"),
                    ("F", "<f4"), ("F2", "<f4")])
B_HIT = np.dtype([("snp1", "<i4"), ("snp2", "<i4"), ("df1", "<i4"), ("df2", "<i4"),
                  ("F", "<f8"), ("F2", "<f8")])

_P = ctypes.c_void_p
_a = None
_b = None


def _ptr(x):
    return None if x is None else x.ctypes.data_as(ctypes.c_void_p)


def have_ref():
    return REF_LIB.exists()


def lib_a():
    global _a
    if _a is None:
        if not REF_LIB.exists():
            raise FileNotFoundError("oracle A not built: python oracle/build_ref.py (needs the reference tree)")
        _a = ctypes.CDLL(str(REF_LIB))
        _a.ref_scan_block.restype = ctypes.c_int64
        _a.ref_scan_block.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _P, ctypes.c_int64, _P, _P, ctypes.c_int]
        _a.ref_phen_stats.restype = None
        _a.ref_phen_stats.argtypes = [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                      ctypes.POINTER(ctypes.c_float)]
    return _a


def lib_b():
    global _b
    if _b is None:
        if not B_LIB.exists():
            subprocess.run(["make", "-C", str(ORACLE), "liboracle.so"], check=True, capture_output=True)
        _b = ctypes.CDLL(str(B_LIB))
        _b.oracle_scan_block.restype = ctypes.c_int64
        _b.oracle_scan_block.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int, _P,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, _P, ctypes.c_int64, _P, _P, _P, _P, _P]
        _b.oracle_unpack.restype = None
        _b.oracle_unpack.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]
        _b.oracle_pack.restype = None
        _b.oracle_pack.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P]
        _b.oracle_permute.restype = None
        _b.oracle_permute.argtypes = [_P, ctypes.c_int, ctypes.c_uint]
    return _b


def phen_stats(phen):
    """perform_scan's float mY/SSY (EpiOpenCL.c:1367-1376)."""
    phen = np.ascontiguousarray(phen, dtype=np.float32)
    m, s = ctypes.c_float(), ctypes.c_float()
    lib_a().ref_phen_stats(_ptr(phen), phen.shape[0], ctypes.byref(m), ctypes.byref(s))
    return m.value, s.value


def ref_scan_block(gpack, nid, phen, block, test="f", safe=0, chunk=128, t1=6.5, t2=10.5, cap=None,
                   dump=False, nthreads=1):
    """Oracle A on one block (start1, size1, start2, size2); block i == j when starts match.
    Returns (hits, total[, counts, means])."""
    gpack = np.ascontiguousarray(gpack, dtype=np.int32)
    phen = np.ascontiguousarray(phen, dtype=np.float32)
    s1, m1, s2, m2 = (int(x) for x in block)
    mY, SSY = phen_stats(phen)
    if cap is None:
        cap = m1 * m2 + 1
    hits = np.zeros(max(cap, 1), dtype=REF_HIT)
    counts = means = None
    if dump:
        counts = np.full((m1, m2, 9), 0xFFFFFFFF, dtype=np.uint32)
        means = np.full((m1, m2, 9), np.nan, dtype=np.float32)
    total = lib_a().ref_scan_block(ord(test), int(safe), int(chunk), _ptr(gpack), nid // 16, nid % 16, nid,
                                   _ptr(phen), mY, SSY, float(t1), float(t2), s1, m1, s2, m2, int(s1 == s2),
                                   _ptr(hits), cap, _ptr(counts), _ptr(means), int(nthreads))
    hits = hits[:min(total, cap)]
    if dump:
        return hits, total, counts.astype(np.int64).astype(np.int32), means
    return hits, total


def oracle_scan_block(codes, phen, block, test="f", safe=0, chunk=128, t1=6.5, t2=10.5, per_pair=False):
    """Oracle B on one block. codes: uint8 (nsnp, nid). Returns (hits, total[, dict])."""
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    phen = np.ascontiguousarray(phen, dtype=np.float32)
    nid = codes.shape[1]
    s1, m1, s2, m2 = (int(x) for x in block)
    cap = m1 * m2 + 1
    hits = np.zeros(cap, dtype=B_HIT)
    out = None
    if per_pair:
        out = {"counts": np.full((m1, m2, 9), -1, dtype=np.int32), "F": np.full((m1, m2), np.nan),
               "F2": np.full((m1, m2), np.nan), "df1": np.full((m1, m2), -1, dtype=np.int32),
               "df2": np.full((m1, m2), -1, dtype=np.int32)}
    total = lib_b().oracle_scan_block(ord(test), int(safe), int(chunk), _ptr(codes), nid, _ptr(phen), float(t1),
                                      float(t2), s1, m1, s2, m2, _ptr(hits), cap,
                                      *([_ptr(out[k]) for k in ("counts", "F", "F2", "df1", "df2")] if out
                                        else [None] * 5))
    hits = hits[:total]
    if per_pair:
        return hits, total, out
    return hits, total


def oracle_unpack(gpack, nid):
    gpack = np.ascontiguousarray(gpack, dtype=np.int32)
    nsnp = gpack.shape[0]
    out = np.zeros((nsnp, nid), dtype=np.uint8)
    lib_b().oracle_unpack(_ptr(gpack), nid, nsnp, nid // 16, nid % 16, _ptr(out))
    return out


def oracle_pack(codes):
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    nsnp, nid = codes.shape
    npack1 = nid // 16 + (1 if nid % 16 else 0)
    out = np.zeros((nsnp, npack1), dtype=np.int32)
    lib_b().oracle_pack(_ptr(codes), nid, nsnp, _ptr(out))
    return out


def oracle_permute(phen, seed):
    p = np.array(phen, dtype=np.float32, copy=True)
    lib_b().oracle_permute(_ptr(p), p.shape[0], int(seed))
    return p


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
