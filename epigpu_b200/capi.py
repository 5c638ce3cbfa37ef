"""ctypes binding of libepigpu.so (include/epigpu.h).

The library is built in-tree (python -m epigpu_b200.build); importing this module without
it raises, there is no fallback implementation.
"""
import ctypes
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "libepigpu.so"

EPI_OK = 0
EPI_E_INVALID = 1
EPI_E_CUDA = 2
EPI_E_NOMEM = 3
EPI_E_OVERFLOW = 4
EPI_E_STATE = 5
EPI_E_TIMEOUT = 6
EPI_E_NODEVICE = 7
EPI_E_UNSUPPORTED = 8

FORM_AUTO, FORM_POPC, FORM_TENSOR = 0, 1, 2
DEBUG_STALL = 1

# Functions include/epigpu.h declares (checked by the CPU tests).
EXPORTS = (
    "epi_default_opts", "epi_open", "epi_close", "epi_strerror", "epi_last_error",
    "epi_device_info", "epi_load_packed", "epi_set_traits", "epi_set_phenotype", "epi_scan",
    "epi_scan_dump", "epi_last_timing", "epi_scan_config", "epi_get_stream", "epi_scan_block_noalloc", "epi_permute_phenotype",
)


class Hit(ctypes.Structure):
    """The reference's `table` row (src/id4117.h:14-21)."""
    _fields_ = [("snp1", ctypes.c_int32), ("snp2", ctypes.c_int32), ("df1", ctypes.c_int32),
                ("df2", ctypes.c_int32), ("F", ctypes.c_float), ("F2", ctypes.c_float)]


class Block(ctypes.Structure):
    _fields_ = [("start1", ctypes.c_int32), ("size1", ctypes.c_int32), ("start2", ctypes.c_int32),
                ("size2", ctypes.c_int32)]


class ScanOpts(ctypes.Structure):
    _fields_ = [("test", ctypes.c_int32), ("safe", ctypes.c_int32), ("chunk", ctypes.c_int32),
                ("t1", ctypes.c_float), ("t2", ctypes.c_float), ("form", ctypes.c_int32),
                ("report_trait", ctypes.c_int32), ("wait_limit_ms", ctypes.c_int32), ("debug", ctypes.c_int32),
                ("no_graph", ctypes.c_int32), ("tile_config", ctypes.c_int32), ("reserved", ctypes.c_int32 * 5)]


HIT_DTYPE = np.dtype([("snp1", "<i4"), ("snp2", "<i4"), ("df1", "<i4"), ("df2", "<i4"),
                      ("F", "<f4"), ("F2", "<f4")])

_P = ctypes.c_void_p
_SIGS = {
    "epi_default_opts": (None, [ctypes.POINTER(ScanOpts)]),
    "epi_open": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(_P)]),
    "epi_close": (ctypes.c_int, [_P]),
    "epi_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "epi_last_error": (ctypes.c_char_p, [_P]),
    "epi_device_info": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "epi_load_packed": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "epi_set_traits": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.c_int32, _P]),
    "epi_set_phenotype": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.c_int32]),
    "epi_scan": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.POINTER(ScanOpts), _P, ctypes.c_int64,
                                ctypes.POINTER(ctypes.c_int64), _P, _P, _P, _P]),
    "epi_scan_dump": (ctypes.c_int, [_P, ctypes.POINTER(Block), ctypes.POINTER(ScanOpts), ctypes.c_int32,
                                     _P, _P, _P, _P, _P]),
    "epi_last_timing": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
    "epi_get_stream": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    "epi_scan_config": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_int32]),
    "epi_scan_block_noalloc": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _P, ctypes.POINTER(Block),
                                              ctypes.POINTER(ScanOpts), _P, ctypes.c_int64, _P, _P, _P]),
    "epi_permute_phenotype": (None, [_P, ctypes.c_int32, ctypes.c_uint32]),
}

_lib = None


def load(path=None):
    """Loads libepigpu.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise OSError("libepigpu.so not built (%s): run `python -m epigpu_b200.build`" % p)
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class EpiError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (status %d): %s" % (load().epi_strerror(status).decode(), status, message))
        self.status = status


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def default_opts(test="f", safe=0, chunk=128, t1=6.5, t2=10.5, form=FORM_AUTO, report_trait=0, wait_limit_ms=0,
                 debug=0, no_graph=0, tile_config=0):
    o = ScanOpts()
    load().epi_default_opts(ctypes.byref(o))
    o.test = ord(test) if isinstance(test, str) else int(test)
    o.safe = int(safe)
    o.chunk = int(chunk)
    o.t1 = float(t1)
    o.t2 = float(t2)
    o.form = int(form)
    o.report_trait = int(report_trait)
    o.wait_limit_ms = int(wait_limit_ms)
    o.debug = int(debug)
    o.no_graph = int(no_graph)
    o.tile_config = int(tile_config)
    return o


def blocks_array(blocks):
    arr = (Block * max(len(blocks), 1))()
    for i, b in enumerate(blocks):
        arr[i] = Block(*[int(x) for x in b])
    return arr


class Context:
    """One device context (epi_open/epi_close)."""

    def __init__(self, device=0):
        self.lib = load()
        h = ctypes.c_void_p()
        st = self.lib.epi_open(int(device), ctypes.byref(h))
        if st != EPI_OK:
            raise EpiError(st, "epi_open(%d)" % device)
        self.h = h

    def close(self):
        if self.h:
            self.lib.epi_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != EPI_OK:
            raise EpiError(st, "%s: %s" % (what, self.lib.epi_last_error(self.h).decode()))

    def device_info(self):
        name = ctypes.create_string_buffer(256)
        sms = ctypes.c_int32()
        self._check(self.lib.epi_device_info(self.h, name, 256, ctypes.byref(sms)), "epi_device_info")
        return name.value.decode(), sms.value

    def load_packed(self, gpack, nid):
        gpack = np.ascontiguousarray(gpack, dtype=np.int32)
        npack, remain = nid // 16, nid % 16
        nsnp = gpack.shape[0]
        self._check(self.lib.epi_load_packed(self.h, _ptr(gpack), nid, nsnp, npack, remain), "epi_load_packed")

    def set_traits(self, y, valid=None):
        """y: (nid,) or (nid, T) float32; valid: same shape bool/uint8 or None (-9 = missing)."""
        y = np.asarray(y, dtype=np.float32)
        if y.ndim == 1:
            y = y[:, None]
        nid, T = y.shape
        yc = np.asfortranarray(y)
        vc = None
        if valid is not None:
            v = np.asarray(valid).astype(np.uint8)
            if v.ndim == 1:
                v = v[:, None]
            vc = np.asfortranarray(v)
        self._check(self.lib.epi_set_traits(self.h, _ptr(yc), nid, T, _ptr(vc)), "epi_set_traits")

    def set_phenotype(self, phen, safe=0):
        phen = np.ascontiguousarray(phen, dtype=np.float32)
        self._check(self.lib.epi_set_phenotype(self.h, _ptr(phen), phen.shape[0], int(safe)), "epi_set_phenotype")

    def scan(self, blocks, opts, cap=1 << 20, ntraits=1, want_blocks=False, want_traits=False):
        """Returns (hits structured array, total, extras dict)."""
        barr = blocks_array(blocks)
        # the library writes the first min(total, cap) rows only: no zero fill (24 MB at the
        # default capacity, most of a small scan's host time)
        hits = np.empty(max(cap, 1), dtype=HIT_DTYPE)
        nh = ctypes.c_int64()
        hb = np.empty(max(cap, 1), dtype=np.int32) if want_blocks else None
        ht = np.empty(max(cap, 1), dtype=np.int32) if want_traits else None
        mf = np.zeros(ntraits, dtype=np.float32)
        mf2 = np.zeros(ntraits, dtype=np.float32)
        st = self.lib.epi_scan(self.h, ctypes.cast(barr, ctypes.c_void_p), len(blocks), ctypes.byref(opts),
                               _ptr(hits), cap, ctypes.byref(nh), _ptr(hb), _ptr(ht), _ptr(mf), _ptr(mf2))
        if st not in (EPI_OK, EPI_E_OVERFLOW):
            self._check(st, "epi_scan")
        n = min(nh.value, cap)
        extras = {"max_f": mf, "max_f2": mf2, "status": st}
        if want_blocks:
            extras["block"] = hb[:n]
        if want_traits:
            extras["trait"] = ht[:n]
        return hits[:n], nh.value, extras

    def scan_dump(self, block, opts, trait=0):
        size1, size2 = int(block[1]), int(block[3])
        np_ = size1 * size2
        counts = np.full((size1, size2, 9), -1, dtype=np.int32)
        F = np.full((size1, size2), np.nan, dtype=np.float32)
        F2 = np.full((size1, size2), np.nan, dtype=np.float32)
        d1 = np.full((size1, size2), -1, dtype=np.int32)
        d2 = np.full((size1, size2), -1, dtype=np.int32)
        b = Block(*[int(x) for x in block])
        if np_:
            self._check(self.lib.epi_scan_dump(self.h, ctypes.byref(b), ctypes.byref(opts), int(trait),
                                               _ptr(counts), _ptr(F), _ptr(F2), _ptr(d1), _ptr(d2)),
                        "epi_scan_dump")
        return {"counts": counts, "F": F, "F2": F2, "df1": d1, "df2": d2}

    def scan_config(self):
        """The form and kernel variant of the last scan and how the variant was chosen."""
        buf = ctypes.create_string_buffer(512)
        self._check(self.lib.epi_scan_config(self.h, buf, 512), "epi_scan_config")
        return buf.value.decode()

    def stream_handle(self):
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        h = ctypes.c_void_p()
        self._check(self.lib.epi_get_stream(self.h, ctypes.byref(h)), "epi_get_stream")
        return h.value or 0

    def last_timing(self):
        """(kernel ms, pair tests, kernel launches, form) of the last scan."""
        ms = ctypes.c_double()
        pairs = ctypes.c_int64()
        nl = ctypes.c_int32()
        form = ctypes.c_int32()
        self._check(self.lib.epi_last_timing(self.h, ctypes.byref(ms), ctypes.byref(pairs), ctypes.byref(nl),
                                             ctypes.byref(form)), "epi_last_timing")
        return ms.value, pairs.value, nl.value, form.value


def permute_phenotype(phen, seed):
    """src/main.c:336-348 on a copy of `phen` (glibc srand/rand)."""
    p = np.array(phen, dtype=np.float32, copy=True)
    load().epi_permute_phenotype(_ptr(p), p.shape[0], int(seed))
    return p
