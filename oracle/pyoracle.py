"""Test infrastructure only: ctypes bindings of the C restatement (oracle/restate.c).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the checker.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "librestate.so")
HIST = 802

CELL_DTYPE = np.dtype([("hyperscore", "<f4"), ("psid", "<i4"), ("idxoffset", "<u2"),
                       ("sharedions", "<u2"), ("totalions", "<u2"), ("pad", "<u2")])
RESULT_DTYPE = np.dtype([
    ("cpsms", "<i4"), ("status", "<i4"), ("top", CELL_DTYPE), ("maxhyp", "<i4"),
    ("mu", "<i4"), ("beta", "<i4"), ("stt1", "<i4"), ("end1", "<i4"), ("pad1", "<i4"),
    ("slope", "<f8"), ("icpt", "<f8"), ("e_x", "<f8"), ("e_fp64", "<f8"),
    ("heap_size", "<i4"), ("pad2", "<i4"), ("heap", CELL_DTYPE, (63,)),
])
CAND_DTYPE = np.dtype([("ixx", "<u2"), ("bc", "<u2"), ("yc", "<u2"), ("pad", "<u2"), ("psid", "<i4"),
                       ("ibc", "<u4"), ("iyc", "<u4"), ("h", "<f4")])


class _Len(C.Structure):
    _fields_ = [("peplen", C.c_uint32), ("npep", C.c_uint32), ("speclen", C.c_uint32),
                ("mass", C.c_void_p), ("bA", C.c_void_p), ("iA", C.c_void_p)]


class _Par(C.Structure):
    _fields_ = [("dM", C.c_double), ("dF", C.c_uint32), ("scale", C.c_uint32), ("max_mass", C.c_double),
                ("min_shp", C.c_uint32), ("min_cpsm", C.c_uint32), ("heap_cap", C.c_int32),
                ("expect_max", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-s", "-C", HERE, "_ref/librestate.so"], check=True)
        _lib = C.CDLL(LIB)
        assert C.sizeof(_Par) == 48
        assert RESULT_DTYPE.itemsize == 88 + 63 * 16, RESULT_DTYPE.itemsize
    return _lib


def heap_capacity(topmatches: int) -> int:
    """Capacity of the reference's top-K heap for a ``topmatches`` setting."""
    import math
    num = 1 if topmatches == 0 else topmatches
    num = int(math.floor(math.log2(num) + 0.999))
    return (1 << num) - 1


class Params:
    def __init__(self, dM=10.0, dF=5, scale=100, max_mass=5000.0, min_shp=4, min_cpsm=4, topmatches=5,
                 expect_max=1e300):
        self.dM, self.dF, self.scale, self.max_mass = dM, dF, scale, max_mass
        self.min_shp, self.min_cpsm, self.topmatches, self.expect_max = min_shp, min_cpsm, topmatches, expect_max

    def c(self):
        return _Par(self.dM, self.dF, self.scale, self.max_mass, self.min_shp, self.min_cpsm,
                    heap_capacity(self.topmatches), self.expect_max)


def _lens(lengths):
    arr = (_Len * len(lengths))()
    keep = []
    for i, x in enumerate(lengths):
        m = np.ascontiguousarray(x["mass"], dtype=np.float32)
        b = np.ascontiguousarray(x["bA"], dtype=np.uint32)
        a = np.ascontiguousarray(x["iA"], dtype=np.uint32)
        keep += [m, b, a]
        arr[i] = _Len(x["L"], x["N"], x["speclen"], m.ctypes.data, b.ctypes.data, a.ctypes.data)
    return arr, keep


def lgfact() -> np.ndarray:
    out = np.zeros(81, np.float64)
    lib().rs_lgfact(out.ctypes.data_as(C.c_void_p))
    return out


def search(lengths, q, params: Params, hist: bool = False, nthreads: int | None = None):
    """Run the restatement over a QueryBatch; returns (results, hist or None)."""
    L = lib()
    arr, keep = _lens(lengths)
    n = q.n
    out = np.zeros(n, RESULT_DTYPE)
    h = np.zeros((n, HIST), np.uint32) if hist else None
    idx = np.ascontiguousarray(q.idx, np.uint32)
    moz = np.ascontiguousarray(q.moz, np.int32)
    it = np.ascontiguousarray(q.intn, np.int32)
    pr = np.ascontiguousarray(q.prec, np.float32)
    dm = None
    if q.dM is not None:
        dm = np.where(np.isnan(q.dM), params.dM, q.dM).astype(np.float64)
    par = params.c()
    rc = L.rs_search(arr, C.c_int(len(lengths)), idx.ctypes.data_as(C.c_void_p), moz.ctypes.data_as(C.c_void_p),
                     it.ctypes.data_as(C.c_void_p), pr.ctypes.data_as(C.c_void_p),
                     None if dm is None else dm.ctypes.data_as(C.c_void_p), C.c_int(n), C.byref(par),
                     out.ctypes.data_as(C.c_void_p), None if h is None else h.ctypes.data_as(C.c_void_p),
                     C.c_int(nthreads or os.cpu_count() or 1))
    if rc != 0:
        raise RuntimeError(f"rs_search failed: {rc}")
    return out, h


def candidates(lengths, moz, intn, prec, dM, params: Params, cap=1 << 22):
    L = lib()
    arr, keep = _lens(lengths)
    out = np.zeros(cap, CAND_DTYPE)
    moz = np.ascontiguousarray(moz, np.int32)
    intn = np.ascontiguousarray(intn, np.int32)
    par = params.c()
    L.rs_candidates.restype = C.c_int64
    n = L.rs_candidates(arr, C.c_int(len(lengths)), moz.ctypes.data_as(C.c_void_p), intn.ctypes.data_as(C.c_void_p),
                        C.c_int(len(moz)), C.c_float(prec), C.c_double(dM), C.byref(par),
                        out.ctypes.data_as(C.c_void_p), C.c_int64(cap))
    if n < 0 or n > cap:
        raise RuntimeError("candidate buffer too small")
    return out[:n]


def tailfit(hist802, cpsms: int, maxhyp: int):
    L = lib()
    r = np.zeros(1, RESULT_DTYPE)
    h = np.ascontiguousarray(hist802, np.float64)
    L.rs_tailfit(h.ctypes.data_as(C.c_void_p), C.c_int32(cpsms), C.c_int32(maxhyp), r.ctypes.data_as(C.c_void_p))
    return r[0]


def window(length, prec: float, dM: float):
    L = lib()
    arr, keep = _lens([length])
    lo, hi = C.c_int32(), C.c_int32()
    L.rs_window(arr, C.c_float(prec), C.c_double(dM), C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def traffic(lengths, q, params: Params):
    """Per-spectrum (in-window ion ids read, distinct probed bins) summed over lengths."""
    L = lib()
    arr, keep = _lens(lengths)
    ids = np.zeros(q.n, np.int64)
    bins = np.zeros(q.n, np.int64)
    par = params.c()
    a, b = C.c_int64(), C.c_int64()
    for i in range(q.n):
        s, e = int(q.idx[i]), int(q.idx[i + 1])
        moz = np.ascontiguousarray(q.moz[s:e], np.int32)
        dm = params.dM if q.dM is None or np.isnan(q.dM[i]) else float(q.dM[i])
        L.rs_traffic(arr, C.c_int(len(lengths)), moz.ctypes.data_as(C.c_void_p), C.c_int(e - s),
                     C.c_float(q.prec[i]), C.c_double(dm), C.byref(par), C.byref(a), C.byref(b))
        ids[i], bins[i] = a.value, b.value
    return ids, bins


def pickpeaks(seg, size, mz, intn, base_int=100000, min_int=1000, qalen=100):
    """Peak picking of raw spectra (rs_pickpeaks per spectrum, on copies of mz/intn):
    returns (idx[n+1], mz, intn) of the kept peaks."""
    L = lib()
    L.rs_pickpeaks.restype = C.c_int
    mz = np.ascontiguousarray(mz, dtype=np.int32).copy()
    intn = np.ascontiguousarray(intn, dtype=np.int32).copy()
    n = len(size)
    idx = np.zeros(n + 1, np.uint32)
    out_m, out_i = [], []
    for s in range(n):
        a, b = int(seg[s]), int(seg[s + 1])
        S = min(int(size[s]), b - a)
        m, i = mz[a:b], intn[a:b]                       # views: sorted and scaled in place
        k = L.rs_pickpeaks(m.ctypes.data_as(C.c_void_p), i.ctypes.data_as(C.c_void_p), C.c_int(b - a), C.c_int(S),
                           C.c_int32(base_int), C.c_int32(min_int), C.c_int(qalen))
        out_m.append(m[b - a - k:].copy())
        out_i.append(i[b - a - k:].copy())
        idx[s + 1] = idx[s] + k
    cat = lambda xs: np.concatenate(xs).astype(np.int32) if xs else np.zeros(0, np.int32)
    return idx, cat(out_m), cat(out_i)
