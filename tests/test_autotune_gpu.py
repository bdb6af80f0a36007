"""The batched path's launch shape and its autotuner (gx_workspace_set_tiles, gx_autotune):
every candidate shape gives byte-identical results on a multi-block workload, the tuner
keeps the fastest of the candidates it timed, a second call for the same workload shape
takes the cached choice, and invalid shapes are refused.  The shapes include the pipelined
kernel (two scorecard tiles per CTA), which takes the spectra with the 8-byte scorecard while
the batched kernel takes the 12-byte ones in the same search."""

import numpy as np
import pytest

from conftest import MULTIBLOCK, concat_queries, has_gpu, multiblock_index, multiblock_queries

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    import gicops_b200 as gx
    H = multiblock_index(2)
    q = concat_queries(multiblock_queries(H, 300, seed=71, window="mixed"), multiblock_queries(H, 200, seed=72))
    dev = gx.DeviceIndex(H, 0)
    s = gx.Searcher(dev, q.n, len(q.moz))
    p = gx.SearchParams(dM=MULTIBLOCK["dM"], expect_max=20.0)
    d = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(d) for k, v in
         dict(idx=q.idx.view(np.int32), moz=q.moz, intn=q.intn, prec=q.prec, charge=q.charge.astype(np.int32),
              dM=np.where(np.isnan(q.dM), p.dM, q.dM)).items()}
    qd = dict(nspec=q.n, npeaks=len(q.moz), **{k: v.data_ptr() for k, v in t.items()})
    return gx, torch, s, q, p, qd, t


def test_every_shape_gives_the_same_results(setup):
    gx, torch, s, q, p, qd, keep = setup
    default = s.tiles
    assert default == {"chunks_per_lane": 2, "ctas_per_sm": 2, "tile": 11264, "sorted": 1, "pipeline": 0}
    ref = s.search(q, p, heap=True, hist=True)
    shapes = [dict(chunks_per_lane=c, ctas_per_sm=k, tile=tile, sorted=so, pipeline=0)
              for c in (1, 2, 3) for k in (1, 2) for tile in (11264, 8448, 4096) for so in (1, 0)]
    shapes += [dict(chunks_per_lane=c, ctas_per_sm=k, tile=11264, sorted=so, pipeline=1)
               for c in (1, 2, 3) for k in (1, 2) for so in (1, 0)]
    for t in shapes:
        s.tiles = t
        r = s.search(q, p, heap=True, hist=True)
        assert r.result.tobytes() == ref.result.tobytes(), t
        assert r.heap.tobytes() == ref.heap.tobytes() and np.array_equal(r.hist, ref.hist), t
    s.tiles = default
    assert len(shapes) == 48


def test_autotune_keeps_the_fastest_and_caches_it(setup):
    gx, torch, s, q, p, qd, keep = setup
    stream = torch.cuda.current_stream().cuda_stream
    r = s.autotune(qd, p, reps=3, use_cache=False, stream=stream)
    assert not r["cached"] and len(r["candidates"]) >= 12
    ms = [c["ms"] for c in r["candidates"]]
    assert all(m > 0 for m in ms)
    fastest = r["candidates"][int(np.argmin(ms))]
    assert r["best"] == {k: fastest[k] for k in r["best"]}
    assert s.tiles == r["best"]
    s.tiles = {"chunks_per_lane": 1, "ctas_per_sm": 1, "tile": 4096, "sorted": 0, "pipeline": 0}
    r2 = s.autotune(qd, p, reps=3, use_cache=True, stream=stream)
    assert r2["cached"] and r2["best"] == r["best"] and s.tiles == r["best"]
    # results with the chosen shape equal the default's
    out = s.search(q, p)
    s.tiles = {"chunks_per_lane": 2, "ctas_per_sm": 2, "tile": 11264, "sorted": 1, "pipeline": 0}
    assert s.search(q, p).result.tobytes() == out.result.tobytes()


def test_invalid_shapes_are_refused(setup):
    gx, torch, s, q, p, qd, keep = setup
    for bad in ({"chunks_per_lane": 0, "ctas_per_sm": 2, "tile": 11264, "sorted": 1},
                {"chunks_per_lane": 4, "ctas_per_sm": 2, "tile": 11264, "sorted": 1},
                {"chunks_per_lane": 2, "ctas_per_sm": 3, "tile": 11264, "sorted": 1},
                {"chunks_per_lane": 2, "ctas_per_sm": 2, "tile": 11296, "sorted": 1},
                {"chunks_per_lane": 2, "ctas_per_sm": 2, "tile": 1000, "sorted": 1},
                {"chunks_per_lane": 2, "ctas_per_sm": 2, "tile": 2048, "sorted": 2},
                {"chunks_per_lane": 2, "ctas_per_sm": 2, "tile": 8448, "sorted": 1, "pipeline": 1},
                {"chunks_per_lane": 2, "ctas_per_sm": 2, "tile": 11264, "sorted": 1, "pipeline": 2}):
        with pytest.raises(gx.GxError) as e:
            s.tiles = bad
        assert e.value.code == -3002
    with pytest.raises(gx.GxError) as e:
        s.autotune(qd, gx.SearchParams(dM=MULTIBLOCK["dM"], flags=gx.FLAG_PLAIN))
    assert e.value.code == -3002


def test_graph_replay_equals_direct_launches(setup):
    """The launch sequence captured in a CUDA graph and replayed gives the same records as
    direct launches: on the first (capturing) call, on a replay, after a change of
    parameters (a new capture), through the device entry point on the caller's stream and
    through the host entry point; each replay counts its kernels."""
    gx, torch, s, q, p, qd, keep = setup
    import dataclasses
    import gicops_b200._native as N
    ref = s.search(q, p, heap=True, hist=True)
    p2 = dataclasses.replace(p, topmatches=10, min_shp=5)
    ref2 = s.search(q, p2).result
    d = torch.device("cuda", 0)
    out = torch.empty(q.n * N.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=d)
    stream = torch.cuda.current_stream().cuda_stream
    s.search_device(qd, p, out.data_ptr(), stream=stream)
    torch.cuda.synchronize()
    direct_dev = out.cpu().numpy().copy()
    s.set_graph(True)
    try:
        for _ in range(2):
            r = s.search(q, p, heap=True, hist=True)
            assert r.result.tobytes() == ref.result.tobytes() and r.heap.tobytes() == ref.heap.tobytes()
            assert np.array_equal(r.hist, ref.hist)
        assert s.search(q, p2).result.tobytes() == ref2.tobytes()
        for _ in range(2):
            out.zero_()
            n0 = gx.lib().gx_launch_count()
            s.search_device(qd, p, out.data_ptr(), stream=stream)
            torch.cuda.synchronize()
            assert gx.lib().gx_launch_count() - n0 >= 4
            assert out.cpu().numpy().tobytes() == direct_dev.tobytes()
    finally:
        s.set_graph(False)
