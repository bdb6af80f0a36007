"""GPU query path vs the oracle and vs the reference's captured PSMs.

Bit-exact: candidate counts, histogram bins, top-K heap contents (ids, shared ions,
float hyperscores), the reported top PSM, tail-fit region and the quantized
slope/intercept (mu, beta).  Floating point: e-values within 1e-9 relative (the
only differences allowed come from the device's log10/pow, which may differ from
the host C library in the last bit).
"""

import numpy as np
import pytest

import pyoracle
from conftest import CASES, assert_same, has_gpu, oracle_params, search_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200
    return gicops_b200


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("flags", [0, 1, 2, "piped"], ids=["default", "wide", "plain", "piped"])
def test_gpu_golden(gx, golden, case, flags):
    c = golden(case)
    H, q = c["index"], c["queries"]
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    if flags == "piped":
        s.tiles = dict(s.tiles, pipeline=1)
        flags = 0
    r = s.search(q, search_params(c, flags=flags), heap=True, hist=True)
    ores, ohist = pyoracle.search(H.lengths, q, oracle_params(c), hist=True)
    assert_same(r.result, r.heap, r.hist, ores, ohist, c)
    # no shared-ion count above MAX_SHDPEAKS (80) on the configs: the reference would read
    # past its lgfact table there (utils.h:110, dslim_query.cpp:936); status bit 4 flags it
    assert not np.any(r.result["status"] & 4)
    if flags == 1:
        assert np.all((r.result["status"] & 8) != 0)


def test_gpu_without_optional_outputs(gx, golden):
    c = golden("open_mox")
    dev = gx.DeviceIndex(c["index"], 0)
    s = gx.Searcher(dev, c["queries"].n, len(c["queries"].moz))
    a = s.search(c["queries"], search_params(c))
    b = s.search(c["queries"], search_params(c), heap=True, hist=True)
    assert a.heap is None and a.hist is None
    assert a.result.tobytes() == b.result.tobytes()


@pytest.mark.parametrize("seed", [21, 22])
def test_gpu_random_open_search(gx, seed):
    """Seeded open search (+-500 Da, Met-ox, charge-2 fragments) beyond the fixtures."""
    db = gx.synth.make_database(600, seed=seed)
    H = gx.HostIndex.build(db, maxz=2, mods=[("M", 15.9949, 2)], nmods=2)
    q = gx.synth.make_queries(H.entries_by_len(), 300, seed=seed + 1, charges=(2, 4), frag_charge2=True,
                              keep_p=(0.2, 0.8), noise_mode="fill")
    p = gx.SearchParams(dM=500.0, expect_max=1e300)
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    r = s.search(q, p, heap=True, hist=True)
    ores, ohist = pyoracle.search(H.lengths, q, pyoracle.Params(dM=500.0), hist=True)
    assert_same(r.result, r.heap, r.hist, ores, ohist, None)
    assert not np.any(r.result["status"] & 4)


def test_gpu_topmatches_and_min_shp(gx, golden):
    """Other heap capacities (topmatches 10 -> 15 cells) and shared-peak thresholds."""
    c = golden("open_mox")
    H, q = c["index"], c["queries"]
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    for tm, shp in [(10, 4), (2, 3), (31, 6)]:
        p = gx.SearchParams(dM=500.0, topmatches=tm, min_shp=shp, expect_max=1e300)
        r = s.search(q, p, heap=True, hist=True)
        ores, ohist = pyoracle.search(H.lengths, q, pyoracle.Params(dM=500.0, topmatches=tm, min_shp=shp), hist=True)
        assert_same(r.result, r.heap, r.hist, ores, ohist, None)


def test_gpu_empty_and_degenerate_spectra(gx, golden):
    c = golden("closed_small")
    H = c["index"]
    q = gx.synth.QueryBatch(
        idx=np.array([0, 0, 3, 4, 6], np.uint32),
        moz=np.array([3, 499999, -7, 150000, 100000, 100000], np.int32),   # filtered peaks, one peak, duplicates
        intn=np.array([100, 100, 100, 100000, 5000, 5000], np.int32),
        prec=np.array([1500.0, 1500.0, 100.0, 1200.0], np.float32),
        charge=np.array([2, 2, 2, 2], np.int32), rtime=np.zeros(4, np.float32))
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, 8, 64)
    p = search_params(c)
    r = s.search(q, p, heap=True, hist=True)
    ores, ohist = pyoracle.search(H.lengths, q, oracle_params(c), hist=True)
    assert_same(r.result, r.heap, r.hist, ores, ohist, None)
    # an empty batch is a no-op
    e = gx.synth.QueryBatch(np.zeros(1, np.uint32), np.zeros(0, np.int32), np.zeros(0, np.int32),
                            np.zeros(0, np.float32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    assert s.search(e, p).result.shape == (0,)


def test_gpu_errors_are_status_codes(gx, golden):
    c = golden("closed_small")
    H, q = c["index"], c["queries"]
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, 4, 4096)
    with pytest.raises(gx.GxError) as e:
        s.search(q, search_params(c))                      # more spectra than the workspace
    assert e.value.code == -3004
    with pytest.raises(gx.GxError) as e:
        s.search(q.subset([0]), gx.SearchParams(topmatches=1))   # zero-capacity heap
    assert e.value.code == -3002
    big = gx.synth.QueryBatch(np.array([0, 2000], np.uint32), np.full(2000, 100000, np.int32),
                              np.full(2000, 1000, np.int32), np.array([1500.0], np.float32),
                              np.array([2], np.int32), np.zeros(1, np.float32))
    with pytest.raises(gx.GxError) as e:
        s.search(big, search_params(c))                   # more peaks than a CTA holds
    assert e.value.code == -3051
    # the context stays usable afterwards
    r = s.search(q.subset([0, 1]), search_params(c))
    assert r.result.shape == (2,)


@pytest.mark.parametrize("flags", [0, 1, 2], ids=["default", "wide", "plain"])
def test_gpu_min_cpsm_zero_and_one(gx, golden, flags):
    """min_cpsm 0 acts as 1: spectra that probe bins but get no candidate PSM (a high
    shared-peak threshold) have no e-value; the rest are fitted as usual."""
    c = golden("open_mox")
    H, q = c["index"], c["queries"]
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    for mc in (0, 1):
        p = gx.SearchParams(dM=500.0, min_shp=16, min_cpsm=mc, expect_max=1e300, flags=flags)
        r = s.search(q, p, heap=True, hist=True)
        ores, ohist = pyoracle.search(H.lengths, q, pyoracle.Params(dM=500.0, min_shp=16, min_cpsm=mc), hist=True)
        assert_same(r.result, r.heap, r.hist, ores, ohist, None)
        none = r.result["cpsms"] == 0
        assert none.sum() > 0 and (~none).sum() > 0
        assert np.all((r.result["status"][none] & 1) == 0)
        assert np.all((r.result["status"][~none] & 1) != 0)


@pytest.mark.parametrize("flags", [0, 2], ids=["batched", "plain"])
def test_gpu_spectrum_over_peak_limit_gets_a_flagged_row(gx, golden, flags):
    """A spectrum with more than GX_MAX_PEAKS peaks is not searched: through the device
    entry point (which does not synchronise to read the guard word) its row is zero with
    status GX_STATUS_PEAK_LIMIT, its histogram and heap rows are empty, and the spectra
    around it are searched as usual."""
    import torch
    import gicops_b200._native as N
    from conftest import concat_queries
    c = golden("open_mox")
    H, q0 = c["index"], c["queries"]
    n = 1500
    over = gx.synth.QueryBatch(np.array([0, n], np.uint32), np.arange(20000, 20000 + 5 * n, 5, dtype=np.int32),
                               np.full(n, 3000, np.int32), np.array([1800.0], np.float32), np.array([3], np.int32),
                               np.zeros(1, np.float32))
    q = concat_queries(q0.subset(np.arange(10)), over, q0.subset(np.arange(10, 30)))
    p = search_params(c, flags=flags)
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    d = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(d) for k, v in
         dict(idx=q.idx.view(np.int32), moz=q.moz, intn=q.intn, prec=q.prec).items()}
    out = torch.full((q.n * N.RESULT_DTYPE.itemsize,), 0x5A, dtype=torch.uint8, device=d)   # stale bytes
    heap = torch.full((q.n * p.heap_cap * N.CELL_DTYPE.itemsize,), 0x5A, dtype=torch.uint8, device=d)
    hist = torch.full((q.n * N.HIST_BINS,), 7, dtype=torch.int32, device=d)
    s.search_device(dict(nspec=q.n, npeaks=len(q.moz), **{k: v.data_ptr() for k, v in t.items()}), p,
                    out.data_ptr(), heap.data_ptr(), hist.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    r = out.cpu().numpy().view(N.RESULT_DTYPE)
    assert r["status"][10] == N.STATUS_PEAK_LIMIT
    z = r[10:11].copy()
    z["status"] = 0
    assert not np.any(z.view(np.uint8))
    assert not np.any(hist.cpu().numpy().reshape(q.n, -1)[10])
    assert not np.any(heap.cpu().numpy().reshape(q.n, -1)[10])
    o, oh = pyoracle.search(H.lengths, q0.subset(np.arange(30)), oracle_params(c), hist=True)
    keep = np.r_[0:10, 11:31]
    assert np.array_equal(r["cpsms"][keep], o["cpsms"])
    assert np.array_equal(hist.cpu().numpy().reshape(q.n, -1)[keep].view(np.uint32), oh)
    assert np.count_nonzero(r["status"] & N.STATUS_PEAK_LIMIT) == 1
