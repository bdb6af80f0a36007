"""Device index to a file and back (gx_index_save / gx_index_load): the loaded index holds
the same arrays and gives byte-identical search results; files of another kind, truncated
files and missing files are refused with status codes (checked without a GPU: the header is
read before any device work)."""

import ctypes as C
import os

import numpy as np
import pytest

from conftest import has_gpu, search_params


def test_load_refuses_bad_files(tmp_path):
    import gicops_b200._native as N
    L = N.lib()
    h = C.c_void_p()
    assert L.gx_index_load(os.fsencode(str(tmp_path / "missing.gxidx")), 0, C.byref(h)) == -3006
    bad = tmp_path / "bad.gxidx"
    bad.write_bytes(b"NOTANIDX" + bytes(200))
    assert L.gx_index_load(os.fsencode(str(bad)), 0, C.byref(h)) == -3003
    assert not h.value


@pytest.mark.gpu
def test_save_load_round_trip(golden, tmp_path):
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200 as gx
    c = golden("open_mox")
    H, q = c["index"], c["queries"]
    dev = gx.DeviceIndex(H, 0)
    path = str(tmp_path / "open_mox.gxidx")
    dev.save(path)
    back = gx.DeviceIndex.load(path, 0, host=H)
    assert back.nbytes == dev.nbytes
    for i in range(H.nlen):
        a, b = dev.read_length(i), back.read_length(i)
        assert all(np.array_equal(a[f], b[f]) for f in ("bA", "iA", "iAb", "mass")), i
    p = search_params(c)
    r1 = gx.Searcher(dev, q.n, len(q.moz)).search(q, p, heap=True, hist=True)
    r2 = gx.Searcher(back, q.n, len(q.moz)).search(q, p, heap=True, hist=True)
    assert r1.result.tobytes() == r2.result.tobytes() and r1.heap.tobytes() == r2.heap.tobytes()
    # a truncated copy is refused
    trunc = str(tmp_path / "trunc.gxidx")
    with open(path, "rb") as f, open(trunc, "wb") as g:
        g.write(f.read()[:-100])
    with pytest.raises(gx.GxError) as e:
        gx.DeviceIndex.load(trunc, 0)
    assert e.value.code == -3012
