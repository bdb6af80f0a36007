"""Streamed search of a host batch in chunks (gx_streamer / gx_search_stream) against one
search of the whole batch: the records must be byte-identical, with and without a learned
tail attached, from pinned and from pageable host memory; a chunk holding more peaks than
the streamer's buffers is refused before any work."""

import ctypes as C

import numpy as np
import pytest

from conftest import MULTIBLOCK, concat_queries, has_gpu, multiblock_index, multiblock_queries


def test_stream_rejects_null_arguments():
    import gicops_b200._native as N
    L = N.lib()
    h = C.c_void_p()
    assert L.gx_streamer_create(None, 1024, 0, C.byref(h)) == -3008
    assert L.gx_search_stream(None, None, None, None, None) == -3008
    assert L.gx_streamer_workspace(None) is None


@pytest.fixture(scope="module")
def setup():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import gicops_b200 as gx
    H = multiblock_index(2)
    q = concat_queries(multiblock_queries(H, 400, seed=61, window="mixed"), multiblock_queries(H, 300, seed=62))
    dev = gx.DeviceIndex(H, 0)
    p = gx.SearchParams(dM=MULTIBLOCK["dM"], expect_max=20.0)
    whole = gx.Searcher(dev, q.n, len(q.moz))
    return gx, H, q, dev, p, whole


def _pinned(q, gx):
    import torch
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    return gx.synth.QueryBatch(pin(q.idx), pin(q.moz), pin(q.intn), pin(q.prec), pin(q.charge.astype(np.int32)),
                               q.rtime, None if q.dM is None else pin(q.dM))


@pytest.mark.gpu
@pytest.mark.parametrize("chunk", [128, 333, 4096])
@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
def test_stream_equals_whole_batch(setup, chunk, pinned):
    gx, H, q, dev, p, whole = setup
    ref = whole.search(q, p).result
    st = gx.Streamer(dev, chunk=chunk)
    qq = _pinned(q, gx) if pinned else q
    out, stats = st.search(qq, p, stats=True)
    assert out.tobytes() == ref.tobytes()
    assert stats["chunks"] == (q.n + chunk - 1) // chunk
    assert stats["total_ms"] > 0 and stats["search_ms"] > 0
    assert (out["status"] & 1).sum() > 0.7 * q.n   # +-10 ppm spectra often have < 4 candidate PSMs
    st.close()


@pytest.mark.gpu
def test_stream_with_learned_tail_equals_whole_batch(setup):
    """The model attached to the streamer's workspace is applied per chunk exactly as to
    the whole batch (an untrained model: only the policy's plumbing is checked here)."""
    import gicops_b200.tail as T
    import gicops_b200._native as N
    gx, H, q, dev, p, whole = setup
    m = T.TailModel(0, max_batch=4096, seed=3)
    below = 10 ** 6
    whole.set_tail(m, below)
    st = gx.Streamer(dev, chunk=256)
    st.set_tail(m, below)
    try:
        ref = whole.search(q, p).result
        out = st.search(q, p)
    finally:
        whole.set_tail(None)
    assert out.tobytes() == ref.tobytes()
    assert ((out["status"] & N.STATUS_LEARNED_TAIL) != 0).sum() > 0
    st.close()


@pytest.mark.gpu
def test_stream_refuses_a_chunk_over_its_peak_buffer(setup):
    gx, H, q, dev, p, whole = setup
    st = gx.Streamer(dev, chunk=256, max_peaks=1000)
    with pytest.raises(gx.GxError) as e:
        st.search(q, p)
    assert e.value.code == -3004
    st.close()
