"""gx_search_device_noalloc: the query path for callers that cannot allocate device memory
(a host whose memory pool owns the whole device, a fixed start-up memory budget, or code
where an allocation could block or fail at a bad moment).  It keeps its scratch in a
fixed-size array inside the library instead of a workspace.

Checked here through the C ABI: two calls in a row give the same results as the
allocating entry point (the array keeps the previous call's contents, so the second call
shows that nothing stale leaks through) -- on a golden case, on windows over several
candidate tiles with per-spectrum tolerances (8- and 12-byte scorecards), and with a
spectrum over the peak limit, which both entry points answer with a flagged empty row --
and batches beyond the array's size are refused.
This file is named so that pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest

from conftest import has_gpu, search_params

pytestmark = pytest.mark.gpu


def _dev_queries(q, p, torch, N):
    d = torch.device("cuda", 0)
    t = dict(idx=torch.from_numpy(q.idx.view(np.int32).copy()).to(d), moz=torch.from_numpy(q.moz.copy()).to(d),
             intn=torch.from_numpy(q.intn.copy()).to(d), prec=torch.from_numpy(q.prec.copy()).to(d))
    dm = None
    if q.dM is not None:   # per-spectrum tolerances (Da); NaN takes the batch's
        t["dM"] = torch.from_numpy(np.where(np.isnan(q.dM), p.dM, q.dM).astype(np.float64)).to(d)
        dm = t["dM"].data_ptr()
    cq = N.Queries(q.n, len(q.moz), t["idx"].data_ptr(), t["moz"].data_ptr(), t["intn"].data_ptr(),
                   t["prec"].data_ptr(), None, dm)
    return cq, t


def _case(name, golden, gx):
    """(host index, queries, params) of a parity case."""
    from conftest import MULTIBLOCK, concat_queries, multiblock_index, multiblock_queries
    if name in ("open_mox", "peak_limit"):
        c = golden("open_mox")
        q = c["queries"]
        if name == "peak_limit":   # one spectrum over GX_MAX_PEAKS: not searched, flagged
            n = 1100
            over = gx.synth.QueryBatch(np.array([0, n], np.uint32), np.arange(20000, 20000 + 7 * n, 7, dtype=np.int32),
                                       np.full(n, 5000, np.int32), np.array([1500.0], np.float32),
                                       np.array([2], np.int32), np.zeros(1, np.float32))
            q = concat_queries(q.subset(np.arange(20)), over, q.subset(np.arange(20, 40)))
        return c["index"], q, search_params(c, flags=gx.FLAG_PLAIN)
    # windows over several 8,192-candidate tiles, half the spectra at +-10 ppm
    H = multiblock_index(2)
    q = multiblock_queries(H, 48, seed=51, window="mixed")
    flags = gx.FLAG_PLAIN | (gx.FLAG_WIDE_SCORECARD if name == "multiblock_wide" else 0)
    return H, q, gx.SearchParams(dM=MULTIBLOCK["dM"], expect_max=1e300, flags=flags)


@pytest.mark.parametrize("name", ["open_mox", "multiblock", "multiblock_wide", "peak_limit"])
def test_noalloc_matches_allocating_path(golden, name):
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    import gicops_b200 as gx
    import gicops_b200._native as N

    H, q, p = _case(name, golden, gx)
    dev = gx.DeviceIndex(H, 0)
    ws = gx.Searcher(dev, q.n, len(q.moz))
    cap = p.heap_cap
    cq, keep = _dev_queries(q, p, torch, N)
    cp = p.c()
    d = torch.device("cuda", 0)

    def outputs():
        return (torch.zeros(q.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=d),
                torch.zeros(q.n * cap * N.CELL_DTYPE.itemsize, dtype=torch.uint8, device=d),
                torch.zeros(q.n * N.HIST_BINS, dtype=torch.int32, device=d))

    stream = torch.cuda.current_stream().cuda_stream
    ref = outputs()
    N.check(gx.lib().gx_search_device(dev.handle, ws.handle, C.byref(cq), C.byref(cp), ref[0].data_ptr(),
                                      ref[1].data_ptr(), ref[2].data_ptr(), stream))
    runs = []
    for _ in range(2):
        o = outputs()
        N.check(gx.lib().gx_search_device_noalloc(dev.handle, C.byref(cq), C.byref(cp), o[0].data_ptr(),
                                                  o[1].data_ptr(), o[2].data_ptr(), stream))
        runs.append(o)
    torch.cuda.synchronize()

    rr = ref[0].cpu().numpy().view(N.RESULT_DTYPE)
    assert (rr["status"] & 1).sum() > 0
    if name == "peak_limit":
        assert rr["status"][20] == N.STATUS_PEAK_LIMIT and rr["cpsms"][20] == 0
        assert np.count_nonzero(rr["status"] & N.STATUS_PEAK_LIMIT) == 1
    for o in runs:
        r = o[0].cpu().numpy().view(N.RESULT_DTYPE)
        for f in ("cpsms", "status", "maxhyp", "mu", "beta", "stt1", "end1"):
            assert np.array_equal(r[f], rr[f]), f
        for f in ("psid", "idxoffset", "sharedions", "totalions"):
            assert np.array_equal(r["top"][f], rr["top"][f]), f
        assert np.array_equal(r["top"]["hyperscore"].view(np.uint32), rr["top"]["hyperscore"].view(np.uint32))
        m = (rr["status"] & 1) != 0
        np.testing.assert_allclose(r["e_x"][m], rr["e_x"][m], rtol=1e-9)
        np.testing.assert_allclose(r["e_fp64"][m], rr["e_fp64"][m], rtol=1e-9)
        assert torch.equal(o[1], ref[1]) and torch.equal(o[2], ref[2])


def test_noalloc_rejects_batches_beyond_its_scratch(golden):
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200 as gx
    import gicops_b200._native as N

    c = golden("closed_small")
    dev = gx.DeviceIndex(c["index"], 0)
    nspec = N.NOALLOC_MAX_WINDOWS // dev.host.nlen + 1
    cq = N.Queries(nspec, 0, None, None, None, None, None, None)      # refused before any pointer is read
    cp = search_params(c, flags=gx.FLAG_PLAIN).c()
    rc = gx.lib().gx_search_device_noalloc(dev.handle, C.byref(cq), C.byref(cp), 1, None, None, None)
    assert rc == -3004
    assert b"exceeds the fixed scratch" in gx.lib().gx_last_error()
