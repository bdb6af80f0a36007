"""Device index builder (gx_index_build: fragment ions, CSR and block layout on the GPU)
against the host builder's index uploaded with gx_index_upload: every per-length array
identical (bA, device ids, 16-bit block ids, masses), the device ids equal to the host
iA re-encoded, and identical search results from the two indexes."""

import numpy as np
import pytest

from conftest import CASES, case_index, has_gpu, search_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200
    return gicops_b200


def _encode(iA, speclen):
    e = iA // speclen
    return (2 * e + ((iA - e * speclen) >= speclen // 2)).astype(np.uint32)


def _same_index(gx, kw, db):
    full = gx.HostIndex.build(db, **kw)
    ent = gx.HostIndex.build(db, ions=False, **kw)
    up = gx.DeviceIndex(full, 0)
    dv = gx.DeviceIndex(ent, 0)
    assert up.nbytes == dv.nbytes
    for i, x in enumerate(full.lengths):
        a, b = up.read_length(i), dv.read_length(i)
        for f in ("bA", "iA", "iAb", "mass"):
            assert np.array_equal(a[f], b[f]), (x["L"], f)
        assert np.array_equal(b["bA"], x["bA"]), x["L"]
        assert np.array_equal(b["iA"], _encode(x["iA"].astype(np.int64), x["speclen"])), x["L"]
    return full, up, dv


@pytest.mark.parametrize("maxz,mods,nmods", [(1, (), 0), (2, (("M", 15.9949, 2),), 2),
                                             (3, (("M", 15.9949, 3), ("STY", 79.96633, 1)), 3)])
def test_device_build_equals_host_build(gx, maxz, mods, nmods):
    db = gx.synth.make_database(400, seed=11 + maxz)
    _same_index(gx, dict(maxz=maxz, mods=list(mods), nmods=nmods), db)


def test_device_built_index_searches_identically(gx):
    db = gx.synth.make_database(600, seed=31)
    kw = dict(maxz=2, mods=[("M", 15.9949, 2)], nmods=2)
    H, up, dv = _same_index(gx, kw, db)
    q = gx.synth.make_queries(H.entries_by_len(), 200, seed=32, charges=(2, 4), frag_charge2=True,
                              keep_p=(0.2, 0.8), noise_mode="fill")
    p = gx.SearchParams(dM=500.0, expect_max=1e300)
    a = gx.Searcher(up, q.n, len(q.moz)).search(q, p, heap=True, hist=True)
    b = gx.Searcher(dv, q.n, len(q.moz)).search(q, p, heap=True, hist=True)
    assert a.result.tobytes() == b.result.tobytes()
    assert a.heap.tobytes() == b.heap.tobytes() and np.array_equal(a.hist, b.hist)


@pytest.mark.parametrize("case", CASES)
def test_device_build_of_golden_index(gx, golden, case):
    """The golden cases' indexes (whose host build is pinned to the reference's digests)
    built on the GPU: same arrays as the uploaded host build, same search results."""
    c = golden(case)
    H = c["index"]
    dv = gx.DeviceIndex(case_index(c, ions=False), 0)
    up = gx.DeviceIndex(H, 0)
    for i, x in enumerate(H.lengths):
        a, b = up.read_length(i), dv.read_length(i)
        for f in ("bA", "iA", "iAb", "mass"):
            assert np.array_equal(a[f], b[f]), (case, x["L"], f)
    q = c["queries"]
    a = gx.Searcher(up, q.n, len(q.moz)).search(q, search_params(c), heap=True, hist=True)
    b = gx.Searcher(dv, q.n, len(q.moz)).search(q, search_params(c), heap=True, hist=True)
    assert a.result.tobytes() == b.result.tobytes() and a.heap.tobytes() == b.heap.tobytes()
