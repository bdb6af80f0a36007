"""The C-ABI library: it loads, exports every entry point include/gicops_b200.h
declares, and its host-side checks answer with the reference's status codes (no
GPU work is issued here)."""

import ctypes as C
import os
import re

import numpy as np

import gicops_b200 as gx
import gicops_b200._native as N
import pyoracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "gicops_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gx_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) >= 15
    lib = C.CDLL(N.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(N.EXPORTED)


def test_heap_capacity_matches_reference_rule():
    for t in range(0, 40):
        assert N.lib().gx_heap_capacity(t) == pyoracle.heap_capacity(t)


def test_lgfact_matches_oracle_bits():
    a = np.zeros(81)
    N.lib().gx_lgfact(a.ctypes.data)
    assert np.array_equal(a.view(np.uint64), pyoracle.lgfact().view(np.uint64))


def test_null_arguments_are_rejected():
    L = N.lib()
    h = C.c_void_p()
    assert L.gx_index_upload(None, 1, 500001, 0, C.byref(h)) == -3008
    assert L.gx_workspace_create(None, 10, 10, C.byref(h)) == -3008
    assert L.gx_search_host(None, None, None, None, None, None, None) == -3008
    assert L.gx_search_device(None, None, None, None, None, None, None, None) == -3008
    assert b"null" in L.gx_last_error()


def test_bad_index_descriptions_are_rejected():
    L = N.lib()
    h = C.c_void_p()
    bA = np.zeros(11, np.uint32)
    d = (N.LengthDesc * 1)()
    d[0] = N.LengthDesc(7, 0, 13, 0, None, bA.ctypes.data, None)       # speclen not 2*(L-1)*maxz
    assert L.gx_index_upload(d, 1, 11, 0, C.byref(h)) == -3003
    assert L.gx_index_upload(d, 0, 11, 0, C.byref(h)) == -3002
    assert L.gx_index_upload(d, 65, 11, 0, C.byref(h)) == -3002
    bA[-1] = 5                                                          # bA[last] != npep*speclen
    d[0] = N.LengthDesc(7, 0, 12, 0, None, bA.ctypes.data, None)
    assert L.gx_index_upload(d, 1, 11, 0, C.byref(h)) == -3003


def test_search_params_roundtrip():
    p = gx.SearchParams(dM=500.0, dF=5, topmatches=10)
    c = p.c()
    assert (c.dM, c.dF, c.topmatches, c.scale) == (500.0, 5, 10, 100)
    assert p.heap_cap == 15


def test_merge_and_prep_argument_checks():
    """gx_merge_shards_device and gx_pickpeaks_device reject bad arguments on the host,
    before any device call."""
    L = N.lib()
    p = gx.SearchParams().c()
    dummy = 16   # never dereferenced: every call below fails its host-side checks
    assert L.gx_merge_shards_device(4, 2, 7, None, dummy, dummy, dummy, dummy, C.byref(p), None, dummy, None) == -3008
    assert L.gx_merge_shards_device(4, 0, 7, dummy, dummy, dummy, dummy, dummy, C.byref(p), None, dummy, None) == -3002
    assert L.gx_merge_shards_device(4, 2, 0, dummy, dummy, dummy, dummy, dummy, C.byref(p), None, dummy, None) == -3002
    assert L.gx_merge_shards_device(4, 2, 32, dummy, dummy, dummy, dummy, dummy, C.byref(p), None, dummy, None) == -3002
    p1 = gx.SearchParams(topmatches=1).c()                       # heap capacity 0
    assert L.gx_merge_shards_device(4, 2, 7, dummy, dummy, dummy, dummy, dummy, C.byref(p1), None, dummy, None) == -3002
    assert L.gx_merge_shards_device(4, 2, 7, dummy, dummy, dummy, dummy, dummy, None, None, dummy, None) == -3008
    assert L.gx_pickpeaks_device(1 << 31, dummy, dummy, dummy, dummy, 100000, 1000, 100, dummy, dummy, dummy,
                                 None) == -3004
    assert b"gx_pickpeaks_device" in L.gx_last_error()
